"""A short, self-contained run of the beam step for kernel profiling.

    python -m tertia_b200.profile_case [--layers 256] [--shape cic] [--precision fp32]
                                        [--steps 1]

Builds the 512 x 512 grid of the c1 workload with a shorter box (so that a
profiler capture stays small), the c1 driver beam (bi-Gaussian, 1e6
particles, n_b/n_0 = 0.5) when the box holds it and a weak beam otherwise,
and runs `steps` beam steps eagerly (no graph, so that every kernel is a
separate launch), then synchronises.  Nothing is timed here: the timings
come from the profiler.
"""
from __future__ import annotations

import argparse


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--layers", type=int, default=256)
    ap.add_argument("--shape", default="cic", choices=["cic", "ngp"])
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--steps", type=int, default=1)
    args = ap.parse_args()

    import torch
    from . import workload as wl
    from .abi import QS_SHAPE_CIC, QS_SHAPE_NGP
    from .mesh import Mesh

    w = wl.make_workload("c1", args.precision)
    cfg = w.cfg
    cfg.nx = args.layers
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


if __name__ == "__main__":
    main()
