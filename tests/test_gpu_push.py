"""The GPU plasma push (MoveParticlesLayerSplit replacement) against the
oracle on identical inputs: particle state and deposit cells bit-exact,
deposit sums within the atomic-order tolerance."""
import numpy as np
import pytest

from tertia_b200 import workload as wl
from tertia_b200.abi import (QS_LAYER_P, QS_LAYER_C, QS_F_JX, QS_F_JY, QS_F_JZ, QS_F_DENS,
                             QS_SHAPE_CIC, QS_SHAPE_NGP)
from gpu_helpers import cfg_for

pytestmark = pytest.mark.gpu

DEP = (QS_F_JX, QS_F_JY, QS_F_JZ, QS_F_DENS)


def state(cfg, seed, pscale=0.08, fscale=0.3):
    rng = np.random.default_rng(seed)
    p = wl.front_plasma(cfg, thermal=False)
    n = len(p["y"])
    p["y"] = rng.uniform(0, 1, n)
    p["z"] = rng.uniform(0, 1, n)
    p["px"], p["py"], p["pz"] = (pscale * rng.standard_normal(n) for _ in range(3))
    P = fscale * rng.standard_normal((6, cfg.nz, cfg.ny))
    C = fscale * rng.standard_normal((6, cfg.nz, cfg.ny))
    return p, P, C


def gpu_push(cfg, p, P, C, full):
    from tertia_b200.mesh import Mesh
    with Mesh(cfg) as m:
        m.load_front_plasma(p)
        for c in range(6):
            m.set_layer(QS_LAYER_P, c, P[c])
            m.set_layer(QS_LAYER_C, c, C[c])
        m.move_particles_layer(0, 0, full)
        q = m.get_plasma()
        dep = np.stack([m.get_layer(QS_LAYER_C, f) for f in DEP])
    return q, dep


@pytest.mark.parametrize("shape", [QS_SHAPE_NGP, QS_SHAPE_CIC])
@pytest.mark.parametrize("full", [0, 1])
def test_push_fp64_bitexact(oracle_lib, shape, full):
    cfg = cfg_for("fp64", n=32, layers=4, shape=shape)
    p, P, C = state(cfg, 3 + full + 10 * shape)
    q, dep = gpu_push(cfg, p, P, C, full)
    r = oracle_lib.push_layer(cfg, p["cell"], p["y"], p["z"], p["px"], p["py"], p["pz"], p["w"],
                              P, C, full=bool(full))
    for k in ("y", "z", "px", "py", "pz"):
        assert np.array_equal(q[k], r[k]), k
    assert np.array_equal(q["cell"], r["cell"])
    assert np.array_equal(dep != 0, r["dep"] != 0)      # deposit cells bit-exact
    np.testing.assert_allclose(dep, r["dep"], rtol=1e-12, atol=1e-14)


def thinned(p):
    """The lattice with every seventh particle removed (cells stay grouped in
    ascending order, but not PPC to a cell): the NGP push then takes the
    one-thread-per-particle kernels instead of the one-thread-per-cell
    kernels of the full lattice."""
    keep = np.arange(len(p["y"])) % 7 != 3
    return {k: np.asarray(v)[keep] for k, v in p.items()}


@pytest.mark.parametrize("shape,layout,n", [(QS_SHAPE_NGP, "lattice", 32),
                                            (QS_SHAPE_NGP, "thinned", 32),
                                            (QS_SHAPE_CIC, "lattice", 32),
                                            (QS_SHAPE_CIC, "thinned", 32),
                                            (QS_SHAPE_CIC, "lattice", 40)])
def test_push_fp32_matches_float_oracle(oracle_lib, shape, layout, n):
    """The FP32 kernels factor the divisions and contract to FMA, so they
    match the oracle's float restatement to FP32 rounding; the deposit cells
    (where a particle's current lands) agree exactly.  CIC grids whose ny is
    not a multiple of 32 take the one-thread-per-particle CIC kernel."""
    cfg = cfg_for("fp32", n=n, layers=4, shape=shape)
    p, P, C = state(cfg, 21 + shape)
    if layout == "thinned":
        p = thinned(p)
    f32 = lambda a: np.asarray(a, dtype=np.float32)
    p32 = {k: (f32(v) if k != "cell" else v) for k, v in p.items()}
    q, dep = gpu_push(cfg, {k: np.asarray(v, dtype=np.float64) for k, v in p32.items()},
                      f32(P).astype(np.float64), f32(C).astype(np.float64), 1)
    r = oracle_lib.push_layer(cfg, p32["cell"], p32["y"], p32["z"], p32["px"], p32["py"],
                              p32["pz"], p32["w"], f32(P), f32(C), full=True, precise=True,
                              dtype=np.float32)
    for k in ("px", "py", "pz"):
        np.testing.assert_allclose(q[k], r[k], rtol=2e-6, atol=2e-7)
    for k in ("y", "z"):
        np.testing.assert_allclose(q[k], r[k], rtol=0, atol=2e-6)
    assert np.array_equal(q["cell"], r["cell"])
    assert np.array_equal(dep != 0, r["dep"] != 0)
    np.testing.assert_allclose(dep, r["dep"], rtol=2e-5, atol=1e-6)


def test_push_fp32_close_to_fp64_oracle(oracle_lib):
    cfg = cfg_for("fp32", n=32, layers=4)
    p, P, C = state(cfg, 5)
    q, dep = gpu_push(cfg, p, P, C, 1)
    r = oracle_lib.push_layer(cfg, p["cell"], p["y"], p["z"], p["px"], p["py"], p["pz"], p["w"],
                              P, C, full=True)
    for k in ("px", "py", "pz"):
        np.testing.assert_allclose(q[k], r[k], rtol=2e-6, atol=2e-7)
    np.testing.assert_allclose(q["y"], r["y"], atol=2e-6)
