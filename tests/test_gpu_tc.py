"""Split-precision tcgen05 transforms (BF16x3, TF32x3, BF16x6) against the
oracle's FP64 transforms, and a beam step on the tensor-core path."""
import numpy as np
import pytest

from tertia_b200 import workload as wl
from gpu_helpers import cfg_for, rel_l2, run_pair

pytestmark = pytest.mark.gpu

# relative L2 error of one 2-D transform against FP64
TOL = {"bf16x3": 6e-5, "tf32x3": 5e-6, "bf16x6": 5e-6}


@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3", "bf16x6"])
@pytest.mark.parametrize("shape", [(128, 128), (256, 128), (128, 384)])
def test_tc_transform_matches_oracle(oracle_lib, prec, shape):
    from tertia_b200.mesh import Mesh
    nz, ny = shape
    cfg = cfg_for(prec, n=8, layers=2)
    cfg.ny, cfg.nz = ny, nz
    rng = np.random.default_rng(nz + 3 * ny)
    x = rng.standard_normal((3, nz, ny))
    with Mesh(cfg) as m:
        for kz in (0, 1):
            for ky in (0, 1):
                y = m.transform2d(x, kz, ky)
                ref = oracle_lib.transform2d(x, kz, ky)
                err = rel_l2(y, ref)
                print(f"tc transform {prec} {shape} kinds ({kz},{ky}): rel L2 {err:.3e}")
                assert err < TOL[prec], (kz, ky, err)


@pytest.mark.parametrize("prec", ["tf32x3", "bf16x6", "bf16x3"])
def test_tc_step_matches_oracle(oracle_lib, prec):
    cfg = cfg_for(prec, n=128, layers=24, h=0.05, hx=0.1)
    beam = wl.small_beam(cfg, n=20000, sigma_r=0.5, sigma_xi=0.5)
    o, m = run_pair(oracle_lib, cfg, beam, [wl.front_plasma(cfg, seed=2)])
    err = rel_l2(m.onaxis_ex(), o.onaxis_ex())
    print(f"tc step {prec}: on-axis Ex rel L2 {err:.3e}")
    assert np.max(np.abs(o.onaxis_ex())) > 1e-4
    assert err < (5e-3 if prec == "bf16x3" else 5e-4), err
