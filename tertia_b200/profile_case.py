"""A short, self-contained run of the beam step for kernel profiling.

    python -m tertia_b200.profile_case [--layers 256] [--shape cic] [--precision fp32]
                                        [--steps 1] [--adjoint] [--grid N]
                                        [--checkpoint-every K]

Builds the 512 x 512 grid of the c1 workload with a shorter box (so that a
profiler capture stays small), the c1 driver beam (bi-Gaussian, 1e6
particles, n_b/n_0 = 0.5) when the box holds it and a weak beam otherwise,
and runs `steps` beam steps eagerly (no graph, so that every kernel is a
separate launch), then synchronises.  With --adjoint: the 256 x 256 grid of
the c3 workload with `layers` layers, a checkpointed march (every 16 layers)
and one adjoint sweep of the loss sum(hx Ex) over 8 layers of the box.
--grid N replaces the transverse grid by N x N cells of the same size (the
c4 grid is 1024); --checkpoint-every sets the adjoint's checkpoint interval.
Nothing is timed here: the timings come from the profiler.
"""
from __future__ import annotations

import argparse


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--layers", type=int, default=256)
    ap.add_argument("--shape", default="cic", choices=["cic", "ngp"])
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--adjoint", action="store_true")
    ap.add_argument("--grid", type=int, default=0)
    ap.add_argument("--checkpoint-every", type=int, default=16)
    args = ap.parse_args()
    if args.adjoint:
        return adjoint_case(args)

    import torch
    from . import workload as wl
    from .abi import QS_SHAPE_CIC, QS_SHAPE_NGP
    from .mesh import Mesh

    w = wl.make_workload("c1", args.precision)
    cfg = w.cfg
    cfg.nx = args.layers
    if args.grid:
        cfg.ny = cfg.nz = args.grid
    cfg.shape = QS_SHAPE_CIC if args.shape == "cic" else QS_SHAPE_NGP
    cfg.use_graph = 0
    spec = w.beams[0]
    if cfg.nx * cfg.hx > 8.0 * spec.sigma_xi:
        beam = wl.sample_beam(cfg, spec)
    else:
        beam = wl.sample_beam(cfg, wl.BeamSpec(100_000, nb_over_n0=1e-4))
    with Mesh(cfg) as m:
        m.load_beam(beam)
        for _ in range(args.steps):
            m.step()
        torch.cuda.synchronize()
        print(f"profile case: {cfg.ny}x{cfg.nz}x{cfg.nx} {args.shape} {args.precision}, "
              f"{args.steps} step(s), {m.kernel_launches()} kernel launches, "
              f"max|Ex| on axis {abs(m.onaxis_ex()).max():.4f}", flush=True)


def adjoint_case(args):
    import numpy as np
    import torch
    from . import workload as wl
    from .abi import QS_SHAPE_CIC, QS_SHAPE_NGP
    from .mesh import Mesh

    w = wl.make_workload("c3", args.precision)
    cfg = w.cfg
    cfg.nx = args.layers
    if args.grid:
        cfg.ny = cfg.nz = args.grid
    cfg.shape = QS_SHAPE_CIC if args.shape == "cic" else QS_SHAPE_NGP
    cfg.ts = 0.0
    cfg.synchrotron = 0
    cfg.use_graph = 0
    beam = wl.workload_beam(w)
    keep = beam["i"] < cfg.nx - 1
    beam = {k: v[keep] for k, v in beam.items()}
    dloss = np.zeros(cfg.nx)
    lo = cfg.nx // 4
    dloss[lo:lo + 8] = cfg.hx
    with Mesh(cfg) as m:
        m.seed_front_plasma(0)
        m.adjoint_checkpoints(args.checkpoint_every)
        m.load_beam(beam)
        m.move_beam_particles()
        m.move_all_split_layers()
        dw = m.adjoint(dloss)
        torch.cuda.synchronize()
        print(f"profile case: adjoint {cfg.ny}x{cfg.nz}x{cfg.nx} {args.shape} {args.precision}, "
              f"{m.kernel_launches()} kernel launches, max|dL/dw| {float(np.abs(dw).max()):.3e}",
              flush=True)


if __name__ == "__main__":
    main()
