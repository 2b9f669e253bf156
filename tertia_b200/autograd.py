"""torch.autograd harness over the adjoint of the xi-march.

WakeLoss maps the driver's longitudinal charge profile (piecewise-constant
weights of xi-bins, one per bin) to a loss on the on-axis longitudinal wake
field (the reference's Ex): loss = sum_i c_i Ex_onaxis(layer i), e.g. c_i = hx
over a witness window.  Forward: scale every beam particle's weight by its
bin's value, deposit the beam (qs_move_beam_particles) and march
(qs_move_all_split_layers) with layer checkpoints.  Backward: qs_adjoint gives
d loss / d w_p per particle; the bin gradient is sum over the bin of
w0_p d loss / d w_p.

The adjoint differentiates the state the mesh holds, which is that of its
most recent forward.  A backward therefore has to come before the next
forward (or adjoint) on the same mesh: WakeLoss records the mesh's
state_version after its forward and its backward raises if the mesh has
changed since, instead of returning the gradient at another point.  Use one
mesh per loss that is still waiting for its backward.
"""
from __future__ import annotations

import numpy as np
import torch

from .mesh import Mesh


class WakeLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, bin_weights, mesh: Mesh, beam: dict, bins, coeff):
        beta = bin_weights.detach().cpu().double().numpy()
        b = dict(beam)
        b["w"] = np.asarray(beam["w"], dtype=np.float64) * beta[bins]
        mesh.load_beam(b)
        mesh.move_beam_particles()
        mesh.move_all_split_layers()
        ex = mesh.onaxis_ex()
        c = np.asarray(coeff, dtype=np.float64)
        ctx.mesh, ctx.beam, ctx.bins, ctx.coeff = mesh, beam, bins, c
        ctx.nbins = len(beta)
        ctx.version = getattr(mesh, "state_version", None)
        return bin_weights.new_tensor(float(np.dot(c, ex)))

    @staticmethod
    def backward(ctx, grad_out):
        version = getattr(ctx.mesh, "state_version", None)
        if ctx.version is not None and version != ctx.version:
            raise RuntimeError(
                "WakeLoss.backward: the mesh has run other calls (another forward, or an adjoint) "
                "since this loss's forward, so its state is no longer the one this gradient "
                "belongs to; call backward before the next forward on the same mesh, or use "
                "one mesh per pending loss")
        g = float(grad_out)
        dw = ctx.mesh.adjoint(g * ctx.coeff)
        w0 = np.asarray(ctx.beam["w"], dtype=np.float64)
        gb = np.bincount(ctx.bins, weights=w0 * dw, minlength=ctx.nbins)
        return (torch.from_numpy(gb).to(device=grad_out.device, dtype=grad_out.dtype),
                None, None, None, None)


def xi_bins(beam: dict, cfg, nbins: int, lo: float, hi: float) -> np.ndarray:
    """Bin index of every beam particle by its xi position in [lo, hi)
    (absolute, in units of the layer coordinate x = (i + frac) hx)."""
    x = (np.asarray(beam["i"]) + np.asarray(beam["x"])) * cfg.hx
    b = np.floor((x - lo) / (hi - lo) * nbins).astype(np.int64)
    return np.clip(b, 0, nbins - 1)


def wake_loss(bin_weights, mesh, beam, bins, coeff):
    return WakeLoss.apply(bin_weights, mesh, beam, bins, coeff)
