"""The adjoint of the xi-march (qs_adjoint) against central finite differences
of the loss, and the FP32 adjoint against the FP64 adjoint.

The loss is the on-axis longitudinal wake field (the reference's Ex) summed
over a window of layers behind the driver; the parameters are the weights of
xi-bins of the driver's charge profile.  The beam is deposited without moving
(Ts = 0, no synchrotron loss), so every loss evaluation sees the same beam
positions."""
import numpy as np
import pytest
import torch

from tertia_b200 import workload as wl
from tertia_b200.abi import PRECISIONS, QS_SHAPE_CIC, QS_SHAPE_NGP, QsError
from tertia_b200.autograd import wake_loss, xi_bins

pytestmark = pytest.mark.gpu

NBINS = 8


def setup(prec, layers=48, n=32, every=8, shape=QS_SHAPE_NGP, weights=False):
    from tertia_b200.mesh import Mesh
    cfg = wl.small_config(n=n, layers=layers, ts=0.0, synchrotron=0, shape=shape)
    cfg.precision = PRECISIONS[prec]
    beam = wl.small_beam(cfg, n=4000, nb=0.3)
    x = (beam["i"] + beam["x"]) * cfg.hx
    bins = xi_bins(beam, cfg, NBINS, float(x.min()), float(x.max()) + 1e-9)
    m = Mesh(cfg)
    front = wl.front_plasma(cfg, thermal=False)
    if weights:   # unequal particle weights (seeded)
        front["w"] = np.asarray(front["w"]) * np.random.default_rng(5).uniform(
            0.5, 1.5, len(front["w"]))
    m.load_front_plasma(front)
    m.adjoint_checkpoints(every)
    # window: a band of layers in the middle of the box, behind the driver
    coeff = np.zeros(cfg.nx)
    coeff[layers // 4: layers // 2] = cfg.hx
    return cfg, m, beam, bins, coeff


def loss_at(m, beam, bins, coeff, beta):
    return float(wake_loss(torch.tensor(beta, dtype=torch.float64), m, beam, bins, coeff))


def adjoint_grad(m, beam, bins, coeff, beta):
    t = torch.tensor(beta, dtype=torch.float64, requires_grad=True)
    wake_loss(t, m, beam, bins, coeff).backward()
    return t.grad.numpy().copy()


def fd_grad(m, beam, bins, coeff, beta, h=1e-3):
    g = np.zeros(NBINS)
    for b in range(NBINS):
        bp, bm = beta.copy(), beta.copy()
        bp[b] += h
        bm[b] -= h
        g[b] = (loss_at(m, beam, bins, coeff, bp) - loss_at(m, beam, bins, coeff, bm)) / (2 * h)
    return g


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_adjoint_fp64_matches_finite_differences():
    cfg, m, beam, bins, coeff = setup("fp64")
    beta = np.random.default_rng(5).uniform(0.5, 1.5, NBINS)
    g = adjoint_grad(m, beam, bins, coeff, beta)
    fd = fd_grad(m, beam, bins, coeff, beta)
    assert np.linalg.norm(fd) > 0
    assert rel(g, fd) < 1e-4, (g, fd)
    m.close()


def test_adjoint_fp32_close_to_fp64_adjoint():
    beta = np.random.default_rng(6).uniform(0.5, 1.5, NBINS)
    grads = {}
    for prec in ("fp64", "fp32"):
        cfg, m, beam, bins, coeff = setup(prec)
        grads[prec] = adjoint_grad(m, beam, bins, coeff, beta)
        m.close()
    assert rel(grads["fp32"], grads["fp64"]) < 1e-4, grads


def test_adjoint_needs_checkpointed_march():
    cfg, m, beam, bins, coeff = setup("fp64")
    m.load_beam(beam)
    m.move_beam_particles()          # a new beam deposit since the last march
    with pytest.raises(QsError):
        m.adjoint(coeff)
    m.close()


def test_adjoint_checkpoint_interval_does_not_change_gradient():
    beta = np.random.default_rng(7).uniform(0.5, 1.5, NBINS)
    out = []
    for every in (5, 48):
        cfg, m, beam, bins, coeff = setup("fp64", every=every)
        out.append(adjoint_grad(m, beam, bins, coeff, beta))
        m.close()
    assert rel(out[0], out[1]) < 1e-9    # atomic order of the FP64 deposits only


# ---- CIC: the particles also carry the adjoint of their in-cell position,
# and the FP32 path regroups the plasma by cell between checkpoints

def test_cic_adjoint_fp64_matches_finite_differences():
    cfg, m, beam, bins, coeff = setup("fp64", shape=QS_SHAPE_CIC)
    beta = np.random.default_rng(8).uniform(0.5, 1.5, NBINS)
    g = adjoint_grad(m, beam, bins, coeff, beta)
    fd = fd_grad(m, beam, bins, coeff, beta)
    assert np.linalg.norm(fd) > 0
    assert rel(g, fd) < 1e-4, (g, fd)
    m.close()


def test_cic_adjoint_fp32_close_to_fp64_adjoint():
    """FP32 CIC regroups the plasma by cell every second full push; the
    adjoint carries the particle adjoints across those reorderings."""
    beta = np.random.default_rng(9).uniform(0.5, 1.5, NBINS)
    grads = {}
    for prec in ("fp64", "fp32"):
        cfg, m, beam, bins, coeff = setup(prec, shape=QS_SHAPE_CIC)
        grads[prec] = adjoint_grad(m, beam, bins, coeff, beta)
        m.close()
    assert rel(grads["fp32"], grads["fp64"]) < 1e-4, grads


def test_cic_adjoint_fp32_unequal_weights_close_to_fp64_adjoint():
    """Particles of unequal weight: the FP32 march regroups them, weights
    included, by cell; the checkpoints keep each particle's weight with it, so
    that a recomputed segment pushes every particle with its own weight (the
    plain FP64 path keeps the load order)."""
    beta = np.random.default_rng(12).uniform(0.5, 1.5, NBINS)
    grads = {}
    for prec in ("fp64", "fp32"):
        cfg, m, beam, bins, coeff = setup(prec, shape=QS_SHAPE_CIC, weights=True)
        grads[prec] = adjoint_grad(m, beam, bins, coeff, beta)
        m.close()
    assert rel(grads["fp32"], grads["fp64"]) < 1e-4, grads


@pytest.mark.parametrize("prec,tol", [("fp32", 1e-5), ("fp64fft", 1e-12)])
def test_cic_adjoint_from_stored_fields_matches_full_recomputation(prec, tol, monkeypatch):
    """With the field store (the fields each push gathered, kept by the
    checkpointed march) a segment is recomputed by its full pushes alone;
    without it (QS_ADJ_FIELDS=0, read when a handle is created) by the whole
    march; with the store cut to the 16 head layers (QS_ADJ_FIELDS=16) the
    two head segments of the sweep come from it and the third from the
    march.  All three give the same gradient."""
    beta = np.random.default_rng(13).uniform(0.5, 1.5, NBINS)
    grads = []
    for store in ("", "16", "0"):
        if store:
            monkeypatch.setenv("QS_ADJ_FIELDS", store)
        else:
            monkeypatch.delenv("QS_ADJ_FIELDS", raising=False)
        cfg, m, beam, bins, coeff = setup(prec, n=128, layers=32, shape=QS_SHAPE_CIC,
                                          weights=True)
        grads.append(adjoint_grad(m, beam, bins, coeff, beta))
        m.close()
    assert np.linalg.norm(grads[0]) > 0
    assert rel(grads[0], grads[2]) < tol, grads
    assert rel(grads[1], grads[2]) < tol, grads


def test_cic_adjoint_fp64_fft_matches_fp64_adjoint():
    """The FP64 path on FFT transforms regroups the plasma by cell like FP32
    and pushes with FMA; its gradient is the plain FP64 path's to rounding."""
    beta = np.random.default_rng(10).uniform(0.5, 1.5, NBINS)
    grads = {}
    for prec in ("fp64", "fp64fft"):
        cfg, m, beam, bins, coeff = setup(prec, shape=QS_SHAPE_CIC)
        grads[prec] = adjoint_grad(m, beam, bins, coeff, beta)
        m.close()
    assert rel(grads["fp64fft"], grads["fp64"]) < 1e-9, grads


def test_cic_adjoint_fp32_maps_inside_transforms():
    """ny = 128: the recomputed march of the FP32 adjoint runs the maps
    between the halves of its FFT transforms."""
    beta = np.random.default_rng(11).uniform(0.5, 1.5, NBINS)
    grads = {}
    for prec in ("fp64", "fp32"):
        cfg, m, beam, bins, coeff = setup(prec, n=128, layers=32, shape=QS_SHAPE_CIC)
        grads[prec] = adjoint_grad(m, beam, bins, coeff, beta)
        m.close()
    assert rel(grads["fp32"], grads["fp64"]) < 1e-4, grads


def test_cic_adjoint_checkpoint_interval_fp32():
    beta = np.random.default_rng(10).uniform(0.5, 1.5, NBINS)
    out = []
    for every in (5, 48):
        cfg, m, beam, bins, coeff = setup("fp32", every=every, shape=QS_SHAPE_CIC)
        out.append(adjoint_grad(m, beam, bins, coeff, beta))
        m.close()
    assert rel(out[0], out[1]) < 1e-5


def test_wake_loss_with_bin_weights_on_the_gpu():
    """Bin weights that live on the GPU get their gradient on the GPU, equal
    to the gradient of the same weights on the host; a second forward on the
    mesh before the first loss's backward is refused."""
    cfg, m, beam, bins, coeff = setup("fp64", layers=24)
    beta = np.random.default_rng(8).uniform(0.5, 1.5, NBINS)
    g_host = adjoint_grad(m, beam, bins, coeff, beta)
    t = torch.tensor(beta, dtype=torch.float64, device="cuda", requires_grad=True)
    wake_loss(t, m, beam, bins, coeff).backward()
    assert t.grad.device.type == "cuda"
    # two FP64 adjoint sweeps agree to the order of their atomic additions
    assert rel(t.grad.cpu().numpy(), g_host) < 1e-9
    l1 = wake_loss(t, m, beam, bins, coeff)
    wake_loss(t.detach(), m, beam, bins, coeff)
    with pytest.raises(RuntimeError, match="state is no longer"):
        l1.backward()
    m.close()
