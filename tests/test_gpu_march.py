"""Full beam steps (Domain::Step = MoveBeamParticles + MoveAllSplitLayers)
on the GPU against the oracle from identical seeded inputs."""
import numpy as np
import pytest

from tertia_b200 import workload as wl
from tertia_b200.abi import QS_F_EX, QS_F_EY, QS_F_BZ, QS_F_RHOBEAM, QS_F_JXBEAM, QS_SHAPE_CIC
from gpu_helpers import cfg_for, rel_l2, run_pair

pytestmark = pytest.mark.gpu

# relative L2 tolerances of the fields against the FP64 oracle
TOL = {"fp64": 1e-10, "fp64fft": 1e-10, "fp32": 5e-4}


def fields_all(obj, cfg, layers=None):
    layers = range(cfg.nx) if layers is None else layers
    return np.stack([np.stack([obj.get_field3d(f, i) for f in range(6)]) for i in layers])


@pytest.mark.parametrize("prec", ["fp64", "fp64fft", "fp32"])
def test_one_step_matches_oracle(oracle_lib, prec):
    cfg = cfg_for(prec, n=32, layers=48, pspread_x=0.01, pspread_y=0.01, pspread_z=0.01)
    beam = wl.small_beam(cfg, n=6000)
    fronts = [wl.front_plasma(cfg, seed=11)]
    o, m = run_pair(oracle_lib, cfg, beam, fronts)
    e_o, e_m = o.onaxis_ex(), m.onaxis_ex()
    assert np.max(np.abs(e_o)) > 1e-3          # a wake was driven
    assert rel_l2(e_m, e_o) < TOL[prec]
    assert rel_l2(fields_all(m, cfg), fields_all(o, cfg)) < TOL[prec]
    for f in (QS_F_RHOBEAM, QS_F_JXBEAM):
        rb_o = np.stack([o.get_beam_currents(f, i) for i in range(cfg.nx + 1)])
        rb_m = np.stack([m.get_beam_currents(f, i) for i in range(cfg.nx + 1)])
        assert rel_l2(rb_m, rb_o) < (1e-12 if prec.startswith("fp64") else 1e-6)
    po, pm = o.get_plasma(), m.get_plasma()
    assert np.array_equal(pm["cell"], po["cell"])
    for k in ("px", "py", "pz"):
        assert rel_l2(pm[k], po[k]) < TOL[prec] * 10


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_two_steps_beam_phase_space(oracle_lib, prec):
    cfg = cfg_for(prec, n=32, layers=48)
    beam = wl.small_beam(cfg, n=5000, sigma_p=0.01)
    fronts = [wl.front_plasma(cfg, seed=s) for s in (1, 2)]
    o, m = run_pair(oracle_lib, cfg, beam, fronts, steps=2)
    bo, bm = o.get_beam(), m.get_beam()
    for k in ("i", "j", "k"):
        assert np.array_equal(bm[k], bo[k]), k
    # the second push saw the first march's fields
    assert np.max(np.abs(bo["py"] - beam["py"])) > 1e-6
    for k in ("py", "pz"):
        assert rel_l2(bm[k] - beam[k], bo[k] - beam[k]) < TOL[prec] * 10
    for k in ("x", "y", "z", "px"):
        np.testing.assert_allclose(bm[k], bo[k], rtol=1e-9 if prec == "fp64" else 1e-5,
                                   atol=1e-12 if prec == "fp64" else 1e-6)
    assert rel_l2(m.onaxis_ex(), o.onaxis_ex()) < TOL[prec]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_cic_step_matches_oracle(oracle_lib, prec):
    """CIC march (FP32: the one-thread-per-home-cell tile kernel, particles
    moving between cells) against the FP64 oracle."""
    cfg = cfg_for(prec, n=32, layers=32, shape=QS_SHAPE_CIC)
    beam = wl.small_beam(cfg, n=4000)
    o, m = run_pair(oracle_lib, cfg, beam, [wl.front_plasma(cfg, seed=3)])
    assert rel_l2(m.onaxis_ex(), o.onaxis_ex()) < (1e-10 if prec == "fp64" else 5e-4)
    po, pm = o.get_plasma(), m.get_plasma()
    if prec == "fp64":
        assert np.array_equal(pm["cell"], po["cell"])
    else:
        assert np.mean(pm["cell"] == po["cell"]) > 0.999
        assert np.any(po["cell"] != wl.front_plasma(cfg, seed=3)["cell"])   # particles moved


@pytest.mark.parametrize("shape", [0, QS_SHAPE_CIC], ids=["ngp", "cic"])
def test_fp32_maps_inside_the_transforms_match_oracle(oracle_lib, shape):
    """At ny >= 128 the FP32 path applies the Guess / Iterate maps between the
    two halves of its FFT transforms (one kernel per z-mode row)."""
    cfg = cfg_for("fp32", n=128, layers=24, shape=shape, pspread_x=0.01, pspread_y=0.01,
                  pspread_z=0.01)
    beam = wl.small_beam(cfg, n=8000)
    o, m = run_pair(oracle_lib, cfg, beam, [wl.front_plasma(cfg, seed=4)] * 2, steps=2)
    e_o, e_m = o.onaxis_ex(), m.onaxis_ex()
    assert np.max(np.abs(e_o)) > 1e-3
    assert rel_l2(e_m, e_o) < TOL["fp32"]
    assert rel_l2(fields_all(m, cfg, range(0, cfg.nx, 5)), fields_all(o, cfg, range(0, cfg.nx, 5))) \
        < TOL["fp32"]


def test_fine_grained_sequence_matches_march(oracle_lib):
    """qs_begin_march / layer_begin / move_split_layer / layer_end in the
    order of MoveAllSplitLayers give the march's layers."""
    from tertia_b200.mesh import Mesh
    cfg = cfg_for("fp64", n=32, layers=12)
    beam = wl.small_beam(cfg, n=3000)
    front = wl.front_plasma(cfg, seed=4)
    o = oracle_lib.Oracle(cfg)
    o.load_beam(beam)
    o.move_beam_particles()
    o.load_front_plasma(front)
    o.begin_march()
    with Mesh(cfg) as m:
        m.load_beam(beam)
        m.move_beam_particles()
        m.load_front_plasma(front)
        m.begin_march()
        for i in range(cfg.nx - 1, -1, -1):
            o.layer_begin(i, 0)
            m.layer_begin(i, 0)
            o.move_split_layer(i, 0)
            m.move_split_layer(i, 0)
            for f in (QS_F_EX, QS_F_EY, QS_F_BZ):
                assert rel_l2(m.get_layer(1, f), o.get_layer(1, f)) < 1e-10, (i, f)
            o.layer_end(i, 0)
            m.layer_end(i, 0)


def test_graph_replay_equals_eager():
    from tertia_b200.mesh import Mesh
    out = []
    for g in (0, 1):
        cfg = cfg_for("fp64", n=32, layers=24)
        cfg.use_graph = g
        beam = wl.small_beam(cfg, n=3000)
        with Mesh(cfg) as m:
            m.load_beam(beam)
            for s in range(3):
                m.load_front_plasma(wl.front_plasma(cfg, seed=s))
                m.step()
            out.append(m.onaxis_ex())
    assert rel_l2(out[1], out[0]) < 1e-12


def test_zero_beam_gives_zero_fields():
    from tertia_b200.mesh import Mesh
    cfg = cfg_for("fp32", n=32, layers=16)
    with Mesh(cfg) as m:
        m.load_beam(wl.small_beam(cfg, n=10, nb=0.0))
        m.load_front_plasma(wl.front_plasma(cfg, thermal=False))
        m.step()
        assert np.all(m.onaxis_ex() == 0.0)


def test_device_seeding_is_deterministic():
    from tertia_b200.mesh import Mesh
    cfg = cfg_for("fp32", n=32, layers=4, pspread_x=0.01, pspread_y=0.01, pspread_z=0.01)
    with Mesh(cfg) as m:
        m.seed_front_plasma(7)
        a = m.get_plasma()
        m.seed_front_plasma(7)
        b = m.get_plasma()
        m.seed_front_plasma(8)
        c = m.get_plasma()
    assert np.array_equal(a["px"], b["px"])
    assert not np.array_equal(a["px"], c["px"])
    assert abs(np.std(a["py"]) - 0.01) < 1e-3
    assert np.allclose(a["w"], cfg.plasma_density / cfg.ppc)


@pytest.mark.parametrize("prec,tol", [("fp64fft", 1e-12), ("fp32", 1e-5)])
def test_side_streams_and_fused_maps_match_the_sequential_march(prec, tol):
    """Inside a march the last E/B transform of each layer and the plasma
    regrouping run on side streams, and (with the maps between the halves of
    the transforms, ny >= 128) the last corrector kernel of a layer also runs
    the next layer's predictor.  With per-kernel timing on, the same march runs
    strictly in order with a predictor kernel of its own per layer.  Both give
    the same fields and plasma (FP32: to the rounding of its atomic deposits)."""
    from tertia_b200.mesh import Mesh
    cfg = cfg_for(prec, n=128, layers=24, pspread_x=0.01, pspread_y=0.01, pspread_z=0.01)
    beam = wl.small_beam(cfg, n=20000)
    front = wl.front_plasma(cfg, seed=3)
    out = {}
    for timed in (False, True):
        with Mesh(cfg) as m:
            m.profile_enable(timed)
            m.load_beam(beam)
            m.load_front_plasma(front)
            m.step()
            out[timed] = (m.onaxis_ex(), fields_all(m, cfg), m.get_plasma())
            if timed:
                prof = m.profile_read()
                assert sum(n for _, n in prof.values()) > 0   # it did run per kernel
    (e0, f0, p0), (e1, f1, p1) = out[False], out[True]
    assert np.max(np.abs(e1)) > 1e-4
    assert rel_l2(e0, e1) < tol
    assert rel_l2(f0, f1) < tol
    if prec == "fp64fft":
        assert np.array_equal(p0["cell"], p1["cell"])
    else:
        assert np.mean(p0["cell"] == p1["cell"]) > 0.9999
    for k in ("px", "py", "pz"):
        assert rel_l2(p0[k], p1[k]) < tol * 10


@pytest.mark.parametrize("prec,shape", [("fp64", "ngp"), ("fp64", "cic"), ("fp64fft", "cic"),
                                        ("fp32", "cic")])
def test_split_layers_match_oracle(oracle_lib, prec, shape):
    """NxSplit = 2: each layer is marched in two sub-layers of hx/2 with the
    beam currents interpolated between the layers (movepart_splitlayer.cpp:
    561-778, the split weights of :430-445); in FP32 and in FP64 on FFT
    transforms the plasma is regrouped across the splits as well."""
    from tertia_b200.abi import QS_SHAPE_NGP
    cfg = cfg_for(prec, n=32, layers=24, pspread_x=0.01, pspread_y=0.01, pspread_z=0.01)
    cfg.nx_split = 2
    cfg.shape = QS_SHAPE_CIC if shape == "cic" else QS_SHAPE_NGP
    beam = wl.small_beam(cfg, n=6000)
    fronts = [wl.front_plasma(cfg, seed=7)]
    o, m = run_pair(oracle_lib, cfg, beam, fronts)
    e_o, e_m = o.onaxis_ex(), m.onaxis_ex()
    assert np.max(np.abs(e_o)) > 1e-3
    assert rel_l2(e_m, e_o) < TOL[prec]
    assert rel_l2(fields_all(m, cfg), fields_all(o, cfg)) < TOL[prec]
    po, pm = o.get_plasma(), m.get_plasma()
    if prec.startswith("fp64"):
        assert np.array_equal(pm["cell"], po["cell"])
    for k in ("px", "py", "pz"):
        assert rel_l2(pm[k], po[k]) < TOL[prec] * 10


@pytest.mark.parametrize("prec", ["fp64", "fp64fft", "fp32"])
def test_two_corrector_iterations_match_oracle(oracle_lib, prec):
    """nIter = 2 (two predictor-corrector passes before the full push,
    movepart_splitlayer.cpp:561-778) on a 128 x 128 grid, where the FP32 and
    FP64-FFT paths run the maps between the halves of their transforms and
    fuse the next layer's predictor into the last corrector."""
    cfg = cfg_for(prec, n=128, layers=16, pspread_x=0.01, pspread_y=0.01, pspread_z=0.01)
    cfg.n_iter = 2
    cfg.shape = QS_SHAPE_CIC
    beam = wl.small_beam(cfg, n=20000)
    fronts = [wl.front_plasma(cfg, seed=9)]
    o, m = run_pair(oracle_lib, cfg, beam, fronts)
    e_o, e_m = o.onaxis_ex(), m.onaxis_ex()
    assert np.max(np.abs(e_o)) > 1e-3
    assert rel_l2(e_m, e_o) < TOL[prec]
    assert rel_l2(fields_all(m, cfg), fields_all(o, cfg)) < TOL[prec]
    po, pm = o.get_plasma(), m.get_plasma()
    if prec.startswith("fp64"):
        assert np.array_equal(pm["cell"], po["cell"])
    for k in ("px", "py", "pz"):
        assert rel_l2(pm[k], po[k]) < TOL[prec] * 10
