"""The torch.autograd wrapper of the adjoint (tertia_b200/autograd.py) over a
stand-in march that is linear in the beam weights (host only): the bin
scaling of the forward, the per-bin reduction of the backward and the
incoming gradient's scale, checked with torch.autograd.gradcheck."""
import numpy as np
import torch

from tertia_b200.autograd import wake_loss, xi_bins


class LinearMarch:
    """On-axis Ex = A w for the loaded beam weights w; its adjoint A^T."""

    def __init__(self, nx, nb, seed=0):
        self.A = np.random.default_rng(seed).standard_normal((nx, nb))
        self.w = None

    def load_beam(self, b):
        self.w = np.asarray(b["w"], dtype=np.float64).copy()

    def move_beam_particles(self):
        pass

    def move_all_split_layers(self):
        self.ex = self.A @ self.w

    def onaxis_ex(self):
        return self.ex

    def adjoint(self, dloss):
        return self.A.T @ np.asarray(dloss, dtype=np.float64)


class Cfg:
    hx = 0.1


def test_bins_follow_xi():
    beam = {"i": np.array([0, 4, 9, 9]), "x": np.array([0.0, 0.5, 0.2, 0.99])}
    b = xi_bins(beam, Cfg, 4, 0.0, 1.0)
    np.testing.assert_array_equal(b, [0, 1, 3, 3])
    np.testing.assert_array_equal(xi_bins(beam, Cfg, 2, 0.5, 1.0), [0, 0, 1, 1])


def test_gradient_of_the_bin_weights():
    nx, nb, nbins = 12, 40, 5
    rng = np.random.default_rng(1)
    beam = {"w": rng.uniform(0.5, 1.5, nb), "i": rng.integers(0, nx, nb), "x": rng.random(nb)}
    bins = rng.integers(0, nbins, nb)
    coeff = rng.standard_normal(nx)
    march = LinearMarch(nx, nb)
    beta = torch.tensor(rng.uniform(0.5, 1.5, nbins), dtype=torch.float64, requires_grad=True)
    loss = wake_loss(beta, march, beam, bins, coeff)
    # the loss itself: c . A (w0 beta[bins])
    w = beam["w"] * beta.detach().numpy()[bins]
    assert float(loss.detach()) == np.dot(coeff, march.A @ w)
    (3.0 * loss).backward()
    g_expect = 3.0 * np.bincount(bins, weights=beam["w"] * (march.A.T @ coeff), minlength=nbins)
    np.testing.assert_allclose(beta.grad.numpy(), g_expect, rtol=1e-12, atol=1e-12)
    assert torch.autograd.gradcheck(lambda b: wake_loss(b, march, beam, bins, coeff),
                                    (beta.detach().clone().requires_grad_(True),))


class StatefulMarch(LinearMarch):
    """A march whose adjoint depends on the last loaded weights (on-axis
    Ex = A (w * w)), with the state counter of tertia_b200.mesh.Mesh."""

    def __init__(self, nx, nb, seed=0):
        super().__init__(nx, nb, seed)
        self.state_version = 0

    def load_beam(self, b):
        self.state_version += 1
        super().load_beam(b)

    def move_beam_particles(self):
        self.state_version += 1

    def move_all_split_layers(self):
        self.state_version += 1
        self.ex = self.A @ (self.w * self.w)

    def adjoint(self, dloss):
        self.state_version += 1
        return 2.0 * self.w * (self.A.T @ np.asarray(dloss, dtype=np.float64))


def _setup(seed=2):
    nx, nb, nbins = 10, 30, 4
    rng = np.random.default_rng(seed)
    beam = {"w": rng.uniform(0.5, 1.5, nb), "i": rng.integers(0, nx, nb), "x": rng.random(nb)}
    bins = rng.integers(0, nbins, nb)
    coeff = rng.standard_normal(nx)
    return nx, nb, nbins, beam, bins, coeff, rng


def test_gradient_of_a_stateful_march():
    nx, nb, nbins, beam, bins, coeff, rng = _setup()
    march = StatefulMarch(nx, nb)
    beta = torch.tensor(rng.uniform(0.5, 1.5, nbins), dtype=torch.float64, requires_grad=True)
    wake_loss(beta, march, beam, bins, coeff).backward()
    w = beam["w"] * beta.detach().numpy()[bins]
    g_expect = np.bincount(bins, weights=beam["w"] * 2.0 * w * (march.A.T @ coeff),
                           minlength=nbins)
    np.testing.assert_allclose(beta.grad.numpy(), g_expect, rtol=1e-12, atol=1e-12)
    assert beta.grad.device == beta.device


def test_backward_after_another_forward_on_the_same_mesh_raises():
    """Two losses built on one mesh before one backward: the first loss's
    gradient would be taken at the second forward's weights, so it raises."""
    import pytest
    nx, nb, nbins, beam, bins, coeff, rng = _setup(3)
    march = StatefulMarch(nx, nb)
    b1 = torch.tensor(rng.uniform(0.5, 1.5, nbins), dtype=torch.float64, requires_grad=True)
    b2 = torch.tensor(rng.uniform(0.5, 1.5, nbins), dtype=torch.float64, requires_grad=True)
    l1 = wake_loss(b1, march, beam, bins, coeff)
    l2 = wake_loss(b2, march, beam, bins, coeff)
    with pytest.raises(RuntimeError, match="state is no longer"):
        l1.backward()
    l2.backward()                     # the latest forward's backward is fine
    assert b2.grad is not None
    # an adjoint between a forward and its backward moves the state on too
    l3 = wake_loss(b2, march, beam, bins, coeff)
    march.adjoint(coeff)
    with pytest.raises(RuntimeError, match="state is no longer"):
        l3.backward()
