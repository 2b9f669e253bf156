"""Non-uniform plasma (Specie::Density profiles) on the GPU: the seeding
kernel's weights against the oracle's SeedParticles weights, the library's
host evaluation against the oracle's, and a march through a channel with a
longitudinal ramp against the oracle (the density of the spectral maps
follows the phase, also inside a replayed graph)."""
import numpy as np
import pytest

from tertia_b200 import abi
from tertia_b200 import workload as wl
from tertia_b200.abi import density_profile
from gpu_helpers import cfg_for, rel_l2

pytestmark = pytest.mark.gpu


def profiles(cfg):
    xf = cfg.hx * cfg.nx
    ramp = dict(begin=0.0, plateau_begin=xf + 1.0, plateau_end=1e9, end=1e10)
    return [
        density_profile(density=1.3, **ramp),
        density_profile(distribution=abi.DIST_GAUSS_ELLIPSOID, density=2.0, x0=xf, radius=0.4,
                        radius_x=3.0, begin=0.0, end=1e9, delta=0.3, xperiod=2.0),
        density_profile(distribution=abi.DIST_GAUSS_CHANNEL, density=1.0, density1=2.0,
                        delta=0.8, radius=0.3, **ramp),
        density_profile(distribution=abi.DIST_CURVED_CHANNEL, density=1.0, delta=0.9, radius=0.3,
                        xperiod=3.0, y_curvature=0.2, z_curvature=0.1, curvature_begin=0.0,
                        curvature_end=1e9, **ramp),
        density_profile(distribution=abi.DIST_PARALLELEPIPED, density=0.7, x0=xf, radius=0.5,
                        radius_y=0.3),
        density_profile(distribution=abi.DIST_EXPONENTIAL, density=1.0, delta=0.5, begin=0.0,
                        plateau_begin=0.5, plateau_end=xf + 2.0, end=1e9),
        density_profile(distribution=abi.DIST_EMPTY_CHANNEL, density=1.0, delta=0.0, radius=0.25,
                        **ramp),
        density_profile(distribution=abi.DIST_COS_GAUSS, density=1.0, x0=xf + 0.5, radius=0.3,
                        radius_x=2.0, begin=0.0, end=1e9, plateau_end=1e9, xperiod=5.0,
                        delta=0.2),
        density_profile(distribution=abi.DIST_TANH_STEP, density=1.0, x0=xf + 0.3, radius=0.5,
                        radius_x=0.7, begin=0.0, end=1e9),
        density_profile(distribution=abi.DIST_ROD, density=1.0, begin=0.0, end=1e9, radius=0.2,
                        yperiod=0.6, zperiod=0.6, angle_y=0.1),
        density_profile(distribution=abi.DIST_LINEAR_STEP, density=1.0, delta=0.5, begin=0.0,
                        plateau_begin=0.5, plateau_end=xf + 2.0, end=1e9),
        density_profile(distribution=abi.DIST_GRADIENT, density=1.0, delta=4.0, begin=0.0,
                        plateau_begin=0.5, plateau_end=xf + 2.0, end=1e9),
        density_profile(distribution=abi.DIST_PERIODIC, density=1.0, density1=3.0, begin=0.0,
                        plateau_begin=0.2, plateau_end=1e9, end=1e10, xperiod=0.37, delta=0.1),
    ]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_seeded_weights_match_the_oracle(oracle_lib, prec):
    from tertia_b200.mesh import Mesh
    cfg = cfg_for(prec, n=32, layers=4)
    o = oracle_lib.Oracle(cfg)
    with Mesh(cfg) as m:
        for i, prof in enumerate(profiles(cfg)):
            for phase in (0.0, 0.77):
                m.set_density_profile(prof)
                m.set_phase(phase)
                o.set_density_profile(prof)
                o.set_phase(phase)
                m.seed_front_plasma(3)
                p = m.get_plasma()
                want = np.repeat(o.front_weights(), cfg.ppc)
                assert np.array_equal(p["w"] == 0.0, want == 0.0), (i, phase)
                tol = 1e-13 if prec == "fp64" else 1e-7
                np.testing.assert_allclose(p["w"], want, rtol=tol, atol=0, err_msg=str(i))
                assert np.array_equal(p["cell"], np.repeat(np.arange(cfg.ny * cfg.nz), cfg.ppc))
    o.close()


def test_host_density_matches_the_oracle(oracle_lib):
    from tertia_b200.mesh import Mesh
    cfg = cfg_for("fp64", n=32, layers=4)
    rng = np.random.default_rng(4)
    pts = np.stack([rng.uniform(-1, 12, 400), rng.uniform(-1, 1, 400), rng.uniform(-1, 1, 400)], 1)
    with Mesh(cfg) as m:
        for prof in profiles(cfg):
            m.set_density_profile(prof)
            got = np.array([m.plasma_density(*q) for q in pts])
            want = np.array([oracle_lib.density(prof, *q) for q in pts])
            np.testing.assert_allclose(got, want, rtol=1e-14, atol=1e-300)
        m.set_density_profile(None)
        assert m.plasma_density(3.0, 0.1, 0.2) == cfg.plasma_density


def test_periodic_profile_needs_a_period():
    from tertia_b200.mesh import Mesh
    cfg = cfg_for("fp64", n=32, layers=4)
    with Mesh(cfg) as m:
        with pytest.raises(abi.QsError):
            m.set_density_profile(density_profile(distribution=abi.DIST_PERIODIC, xperiod=0.0))


def channel_ramp(cfg):
    # a hollow channel whose density ramps up along x: at the head of the box
    # the on-axis density of the maps differs from the uniform 1
    xf = cfg.hx * cfg.nx
    return density_profile(distribution=abi.DIST_GAUSS_CHANNEL, density=0.5, density1=1.5,
                           delta=0.6, radius=0.4, begin=0.0, plateau_begin=0.0,
                           plateau_end=xf + 4.0, end=1e9)


@pytest.mark.parametrize("prec,shape", [("fp64", abi.QS_SHAPE_NGP), ("fp64", abi.QS_SHAPE_CIC),
                                        ("fp32", abi.QS_SHAPE_CIC)])
def test_channel_march_matches_oracle(oracle_lib, prec, shape):
    from tertia_b200.mesh import Mesh
    cfg = cfg_for(prec, n=32, layers=32, shape=shape, pspread_x=0.01, pspread_y=0.01,
                  pspread_z=0.01)
    beam = wl.small_beam(cfg, n=4000)
    prof = channel_ramp(cfg)
    o = oracle_lib.Oracle(cfg)
    m = Mesh(cfg)
    for h in (o, m):
        h.set_density_profile(prof)
        h.set_phase(0.3)
        h.load_beam(beam)
    m.seed_front_plasma(1)
    front = m.get_plasma()
    assert np.any(front["w"] == 0.0) or np.ptp(front["w"]) > 0
    for s in range(2):
        o.load_front_plasma(front)
        m.load_front_plasma(front)
        o.step()
        m.step()
    assert abs(m.get_phase() - (0.3 + 2 * cfg.ts)) < 1e-15
    e_o, e_m = o.onaxis_ex(), m.onaxis_ex()
    assert np.max(np.abs(e_o)) > 1e-3
    assert rel_l2(e_m, e_o) < (1e-10 if prec == "fp64" else 5e-4)
    # the profile changed the wake: the same particles in uniform-density maps differ
    u = Mesh(cfg)
    u.set_phase(0.3)
    u.load_beam(beam)
    for s in range(2):
        u.load_front_plasma(front)
        u.step()
    assert rel_l2(u.onaxis_ex(), e_o) > 1e-6
    for h in (o, m, u):
        h.close()


def test_graph_follows_a_changing_density():
    """With a ramp the density of the maps changes every step; the captured
    march reads it from device memory, so replay equals eager."""
    from tertia_b200.mesh import Mesh
    out = []
    for g in (0, 1):
        cfg = cfg_for("fp64", n=32, layers=24)
        cfg.use_graph = g
        cfg.ts = 0.5
        beam = wl.small_beam(cfg, n=3000)
        xf = cfg.hx * cfg.nx
        prof = density_profile(density=2.0, begin=xf - 1.0, plateau_begin=xf + 2.0,
                               plateau_end=1e9, end=1e10)
        with Mesh(cfg) as m:
            m.set_density_profile(prof)
            m.load_beam(beam)
            for s in range(3):
                m.load_front_plasma(wl.front_plasma(cfg, seed=s))
                m.step()
                out.append(m.onaxis_ex())
    eager, graph = out[:3], out[3:]
    for a, b in zip(graph, eager):
        assert rel_l2(a, b) < 1e-12
    assert rel_l2(eager[2], eager[1]) > 1e-6
