"""Known-answer tests of the oracle's plasma push (movepart_splitlayer.cpp
:882-1615) and a bit-exact cross-check against an independent numpy
restatement of the same formulas."""
import numpy as np

from tertia_b200 import workload as wl
from tertia_b200.abi import QS_SHAPE_CIC

from refpush import push_ngp


def fields(cfg, rng, scale=0.05):
    return (scale * rng.standard_normal((6, cfg.nz, cfg.ny)),
            scale * rng.standard_normal((6, cfg.nz, cfg.ny)))


def uniform(cfg, e=(0, 0, 0), b=(0, 0, 0)):
    F = np.zeros((6, cfg.nz, cfg.ny))
    for c, v in enumerate(tuple(e) + tuple(b)):
        F[c] = v
    return F


def test_uniform_E_from_rest(oracle_lib):
    """B = 0, p = 0: the two half kicks give p = q2m * hx * E exactly."""
    cfg = wl.small_config(n=16, layers=4)
    p = wl.front_plasma(cfg, thermal=False)
    E = (0.3, -0.2, 0.1)
    F = uniform(cfg, e=E)
    r = oracle_lib.push_layer(cfg, p["cell"], p["y"], p["z"], p["px"], p["py"], p["pz"], p["w"],
                              F, F, full=True)
    hx = cfg.hx
    for comp, e in zip(("px", "py", "pz"), E):
        np.testing.assert_allclose(r[comp], cfg.plasma_q2m * hx * e, rtol=1e-14, atol=0)


def test_uniform_B_preserves_momentum_norm(oracle_lib):
    cfg = wl.small_config(n=16, layers=4)
    rng = np.random.default_rng(3)
    p = wl.front_plasma(cfg, thermal=False)
    n = len(p["y"])
    px, py, pz = (0.05 * rng.standard_normal(n) for _ in range(3))
    F = uniform(cfg, b=(0.4, -0.7, 0.2))
    r = oracle_lib.push_layer(cfg, p["cell"], p["y"], p["z"], px, py, pz, p["w"], F, F, full=True)
    before = np.sqrt(px ** 2 + py ** 2 + pz ** 2)
    after = np.sqrt(r["px"] ** 2 + r["py"] ** 2 + r["pz"] ** 2)
    np.testing.assert_allclose(after, before, rtol=1e-13)


def test_matches_numpy_restatement_bitwise(oracle_lib):
    cfg = wl.small_config(n=32, layers=4)
    rng = np.random.default_rng(11)
    p = wl.front_plasma(cfg, thermal=False)
    n = len(p["y"])
    px, py, pz = (0.03 * rng.standard_normal(n) for _ in range(3))
    y = rng.uniform(0, 1, n)
    z = rng.uniform(0, 1, n)
    P, C = fields(cfg, rng)
    r = oracle_lib.push_layer(cfg, p["cell"], y, z, px, py, pz, p["w"], P, C, full=True)
    ref = push_ngp(cfg, p["cell"], y, z, px, py, pz, p["w"], P, C)
    for k in ("px", "py", "pz", "y", "z"):
        assert np.array_equal(r[k], ref[k]), k
    assert np.array_equal(r["dep_cell"], ref["dep_cell"])
    np.testing.assert_allclose(r["dep"], ref["dep"], rtol=1e-12, atol=1e-15)


def test_particles_keep_their_cell_and_charge_is_conserved(oracle_lib):
    """The live path relinks a particle to GetNyz(jtmp,ktmp) with the outer
    jtmp = j (movepart_splitlayer.cpp:1348-1350, 1507): it keeps its cell
    while its fraction moves.  The deposited charge equals sum w drho0/(1-Vx)."""
    cfg = wl.small_config(n=16, layers=4)
    rng = np.random.default_rng(5)
    p = wl.front_plasma(cfg, thermal=False)
    n = len(p["y"])
    py = 2.0 * np.ones(n)            # fast transverse motion: many cross a boundary
    px = np.zeros(n)
    pz = np.zeros(n)
    F = uniform(cfg)
    r = oracle_lib.push_layer(cfg, p["cell"], p["y"], p["z"], px, py, pz, p["w"], F, F, full=True)
    assert np.array_equal(r["cell"], p["cell"])
    moved = r["dep_cell"] != p["cell"]
    assert moved.any()
    gam = np.sqrt(1 + py ** 2)
    vx_avg = 0.0
    total = np.sum(p["w"] * cfg.plasma_drho0 / (1 - vx_avg))
    np.testing.assert_allclose(r["dep"][3].sum(), total, rtol=1e-13)
    # the fraction is the fractional part of y + dy
    dy = (py / gam) * cfg.hx / cfg.hy
    np.testing.assert_allclose(r["y"], np.mod(p["y"] + dy, 1.0), rtol=0, atol=1e-12)


def test_subcycling_restarts_from_the_seeded_cell(oracle_lib):
    """|dy| > 1 splits the move into ceil(|dy|) sub-steps (:1389-1479), but
    each sub-step adds the OUTER j_jump = j (:1380, :1420) while the inner
    j_jump of :1434 is declared after that statement: the walk restarts from
    the seeded cell.  With y = 1/3 and dy = 4.47 the four unit sub-steps all
    land in cell j+1 and the last 0.47 sub-step lands back in cell j, instead
    of a walk over five cells."""
    cfg = wl.small_config(n=16, layers=4, hx=0.5, h=0.1)
    p = wl.front_plasma(cfg, thermal=False)
    zero = np.zeros(1)
    F = uniform(cfg)
    c0 = int(p["cell"][0])
    j0, k0 = c0 % cfg.ny, c0 // cfg.ny
    r = oracle_lib.push_layer(cfg, p["cell"][:1], p["y"][:1], p["z"][:1], zero,
                              np.array([2.0]), zero, p["w"][:1], F, F, full=False)
    dy = (2.0 / np.sqrt(5.0)) * cfg.hx / cfg.hy
    assert 4 < dy < 5
    rho = r["dep"][3]
    q = p["w"][0] * cfg.plasma_drho0
    assert np.count_nonzero(rho) == 2
    np.testing.assert_allclose(rho[k0, (j0 + 1) % cfg.ny], 4.0 / dy * q, rtol=1e-13)
    np.testing.assert_allclose(rho[k0, j0], (dy - 4.0) / dy * q, rtol=1e-12)
    np.testing.assert_allclose(rho.sum(), q, rtol=1e-14)


def test_cic_conserves_charge_and_relinks(oracle_lib):
    cfg = wl.small_config(n=16, layers=4, shape=QS_SHAPE_CIC)
    rng = np.random.default_rng(8)
    p = wl.front_plasma(cfg, thermal=False)
    n = len(p["y"])
    px, py, pz = (0.2 * rng.standard_normal(n) for _ in range(3))
    P, C = fields(cfg, rng)
    r = oracle_lib.push_layer(cfg, p["cell"], p["y"], p["z"], px, py, pz, p["w"], P, C, full=True)
    assert np.all((r["y"] >= 0) & (r["y"] < 1) & (r["z"] >= 0) & (r["z"] < 1))
    assert not np.array_equal(r["cell"], p["cell"])
    # deposit charge = sum w drho0 / (1 - Vx_avg) recomputed from the push
    assert r["dep"][3].sum() < 0
