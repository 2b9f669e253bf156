"""qs_transform2d_noalloc, the FP64 2-D transform for callers that cannot
allocate device memory, against qs_transform2d_dev of an FP64 handle on the
same device planes.  Two calls in a row with different sizes and kinds, then
the first call again, check that the shared fixed scratch array carries
nothing from one call into the next.  The file name sorts last so that pytest
runs it after every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from gpu_helpers import cfg_for, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-13          # the FP64 transform tolerance of the transform tests


def handle_transform(L, ny, nz, kz, ky, x_dev, torch):
    """The existing entry point: an FP64 handle's qs_transform2d_dev."""
    from tertia_b200.mesh import Mesh
    cfg = cfg_for("fp64", n=8, layers=2)
    cfg.ny, cfg.nz = ny, nz
    out = torch.empty_like(x_dev)
    with Mesh(cfg) as m:
        st = L.qs_transform2d_dev(m._h, kz, ky, x_dev.shape[0], C.c_void_p(x_dev.data_ptr()),
                                  C.c_void_p(out.data_ptr()))
        assert st == 0, L.qs_last_error(m._h).decode()
        m.sync()
    return out


def noalloc_transform(L, ny, nz, kz, ky, x_dev, torch):
    out = torch.full_like(x_dev, float("nan"))
    stream = torch.cuda.current_stream().cuda_stream
    st = L.qs_transform2d_noalloc(kz, ky, ny, nz, x_dev.shape[0], C.c_void_p(x_dev.data_ptr()),
                                  C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    assert st == 0, L.qs_last_error(None).decode()
    torch.cuda.synchronize()
    return out


def test_noalloc_matches_handle_transform_twice():
    import torch
    from tertia_b200.abi import load_library
    L = load_library()
    torch.cuda.set_device(0)
    cases = [(128, 64, 0, 1, 3), (64, 512, 1, 0, 2), (128, 64, 0, 1, 3)]
    for ny, nz, kz, ky, batch in cases:
        rng = np.random.default_rng(ny + 3 * nz + kz)
        x = torch.from_numpy(rng.standard_normal((batch, nz, ny))).cuda()
        got = noalloc_transform(L, ny, nz, kz, ky, x, torch).cpu().numpy()
        want = handle_transform(L, ny, nz, kz, ky, x, torch).cpu().numpy()
        assert np.isfinite(got).all()
        err = rel_l2(got, want)
        assert err < TOL, ((ny, nz, kz, ky), err)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from tertia_b200.abi import QS_ERR_INVALID, load_library
    L = load_library()
    x = torch.zeros((1, 8, 1024), dtype=torch.float64, device="cuda")
    for ny, nz in ((1024, 8), (8, 520), (12, 8)):
        st = L.qs_transform2d_noalloc(0, 0, ny, nz, 1, C.c_void_p(x.data_ptr()),
                                      C.c_void_p(x.data_ptr()), None)
        assert st == QS_ERR_INVALID
        msg = L.qs_last_error(None).decode()
        assert "qs_transform2d_noalloc" in msg
        if ny > 512 or nz > 512:
            assert "512" in msg


def test_noalloc_two_calls_queued_on_a_side_stream():
    """Two calls of different sizes and kinds enqueued back to back on one
    non-default stream with no synchronisation between them: the second
    call's matrix set-up is ordered after the first call's transforms by the
    stream, so both outputs match the handle transform."""
    import torch
    from tertia_b200.abi import load_library
    L = load_library()
    torch.cuda.set_device(0)
    side = torch.cuda.Stream()
    cases = [(128, 64, 0, 1, 2), (64, 256, 1, 1, 3)]
    xs, outs = [], []
    for ny, nz, kz, ky, batch in cases:
        rng = np.random.default_rng(7 * ny + nz + ky)
        xs.append(torch.from_numpy(rng.standard_normal((batch, nz, ny))).cuda())
        outs.append(torch.full_like(xs[-1], float("nan")))
    torch.cuda.synchronize()
    for (ny, nz, kz, ky, batch), x, out in zip(cases, xs, outs):
        st = L.qs_transform2d_noalloc(kz, ky, ny, nz, batch, C.c_void_p(x.data_ptr()),
                                      C.c_void_p(out.data_ptr()), C.c_void_p(side.cuda_stream))
        assert st == 0, L.qs_last_error(None).decode()
    side.synchronize()
    for (ny, nz, kz, ky, batch), x, out in zip(cases, xs, outs):
        want = handle_transform(L, ny, nz, kz, ky, x, torch).cpu().numpy()
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        assert rel_l2(got, want) < TOL, (ny, nz, kz, ky)
