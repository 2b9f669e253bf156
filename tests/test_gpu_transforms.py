"""GPU half-integer transforms (qs_transform2d, the CUDA_WRAP_fourierHalfInteger2D
replacement) against the oracle's FFTW-definition transforms."""
import numpy as np
import pytest

from gpu_helpers import cfg_for, rel_l2

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-13, "fp64fft": 1e-13, "fp32": 2e-6}


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", [(32, 32), (64, 128), (128, 64), (256, 256), (512, 512),
                                   (1024, 256), (2048, 32), (48, 40)])
def test_transform_matches_oracle(oracle_lib, prec, shape):
    from tertia_b200.mesh import Mesh
    nz, ny = shape
    cfg = cfg_for(prec, n=8, layers=2)
    cfg.ny, cfg.nz = ny, nz
    rng = np.random.default_rng(ny * 7 + nz)
    x = rng.standard_normal((5, nz, ny))
    with Mesh(cfg) as m:
        for kz in (0, 1):
            for ky in (0, 1):
                y = m.transform2d(x, kz, ky)
                ref = oracle_lib.transform2d(x, kz, ky)
                assert rel_l2(y, ref) < TOL[prec], (kz, ky, rel_l2(y, ref))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_transform_roundtrip(prec):
    from tertia_b200.mesh import Mesh
    cfg = cfg_for(prec, n=64, layers=2)
    rng = np.random.default_rng(1)
    x = rng.standard_normal((3, 64, 64))
    with Mesh(cfg) as m:
        for kz in (0, 1):
            for ky in (0, 1):
                back = m.transform2d(m.transform2d(x, kz, ky), kz, ky) / (4 * 64 * 64)
                assert rel_l2(back, x) < 10 * TOL[prec]


@pytest.mark.parametrize("shape", [(32, 32), (64, 128), (256, 512), (1024, 1024), (512, 64)])
def test_fp64_fft_transform_matches_oracle(oracle_lib, shape):
    """QS_PREC_FP64_FFT: the FFT kernels of the FP32 path in FP64."""
    from tertia_b200.mesh import Mesh
    nz, ny = shape
    cfg = cfg_for("fp64fft", n=8, layers=2)
    cfg.ny, cfg.nz = ny, nz
    rng = np.random.default_rng(ny * 3 + nz)
    x = rng.standard_normal((3, nz, ny))
    with Mesh(cfg) as m:
        for kz in (0, 1):
            for ky in (0, 1):
                y = m.transform2d(x, kz, ky)
                ref = oracle_lib.transform2d(x, kz, ky)
                assert rel_l2(y, ref) < TOL["fp64fft"], (kz, ky, rel_l2(y, ref))


def test_fp64_fft_rejects_unsupported_sizes():
    from tertia_b200.abi import QS_ERR_UNSUPPORTED, QsError
    from tertia_b200.mesh import Mesh
    cfg = cfg_for("fp64fft", n=48, layers=2)
    with pytest.raises(QsError) as e:
        Mesh(cfg)
    assert e.value.status == QS_ERR_UNSUPPORTED
