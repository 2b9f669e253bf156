#!/usr/bin/env python
"""Benchmark of the quasi-static xi-layer loop: particle-layer pushes/s.

One step = one beam time step of the reference's Domain::Step (step.cpp:24):
driver-beam push + 3-D CIC deposit, then the full xi-march over every layer
(front seeding, Guess, nIter x (push, Iterate), full push, Iterate).
One particle-layer push = one plasma macro-particle carried across one
xi-layer (all nIter+1 sub-pushes counted once): Np * layers per step.

Default workload (N=1): c1 with CIC deposit, 512 x 512 transverse cells, 1024 layers, 4 ppc
(1,048,576 plasma particles per layer), thermal sigma_p = 0.01, 1e6 driver
particles, synthetic seeded inputs.  The field store (6.4 GB) and beam-current
store (2.1 GB) are far larger than L2, so every step streams from HBM.

  python bench.py [--gpus N --steps K --warmup W --precision fp32 --shape cic]
  python bench.py --impl reference     # the reference's CPU path (oracle port)

Under torchrun (N>1) every rank runs an independent replica: the march is
serial in xi and does not shard (replicas only, no collective in the path).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "particle-layer pushes/s"
UNIT = "pushes/s"
CLASSES = ["push_deposit", "transform_gemm", "transform_split", "spectral_maps",
           "beam_spectra", "beam_push", "front_seed", "other", "plasma_regroup"]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c1")
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--shape", default="cic", choices=["cic", "ngp"],
                    help="plasma particle shape: CIC deposit (default) or the reference's "
                         "live NGP path")
    ap.add_argument("--layers", type=int, default=0,
                    help="profiling case: the workload's grid with this many layers and a "
                         "weak 1e5-particle beam (not a bench line)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64-plain comparison")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the c3 adjoint measurement")
    ap.add_argument("--no-next", action="store_true",
                    help="skip the density-profile march and hand-off measurements")
    ap.add_argument("--no-c2", action="store_true", help="skip the c2 precision study")
    ap.add_argument("--no-c4", action="store_true", help="skip the c4 full-form measurement")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target seconds of the bounded CPU sample")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers
def dist_env():
    from tertia_b200.replicas import dist_env as env
    return env()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, interval_ms: int = 100):
        self.device = device
        self.interval_ms = interval_ms
        self.rows = []
        self.first = 0
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", str(self.interval_ms), "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        def reader():
            for line in self.proc.stdout:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    self.rows.append(parts)
        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()
        # nvidia-smi takes a moment to print its first row: wait for it (at
        # most 5 s), so that the samples cover the whole timed region.
        t_end = time.monotonic() + 5.0
        while not self.rows and self.proc.poll() is None and time.monotonic() < t_end:
            time.sleep(0.01)

    def mark(self):
        """Start of the timed region: stop() summarises the rows from here on."""
        self.first = len(self.rows)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = self.rows[self.first:] or self.rows[-1:]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for name, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], p["bf16_tflops"], p.get("bf16_tflops_sustained", p["bf16_tflops"]), \
            "measured"
    except Exception:
        return 6650.0, 1590.0, 1400.0, "fallback"


def traffic_record(kernel: str, workload: str, precision: str):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu
    summary (profiles/traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
        return t.get(f"{kernel}:{workload}:{precision}")
    except Exception:
        return None


def cpu_sample(w, target_s: float):
    """Time the oracle (the reference's FP64 CPU path restated) on a bounded
    sample of the same workload: the full transverse grid, a few layers near
    the front (per-layer cost does not depend on the beam)."""
    import numpy as np
    from oracle import binding as ob
    from tertia_b200 import workload as wl
    cores = os.cpu_count() or 1
    ob.set_threads(cores)

    def run(layers):
        cfg = w.cfg.copy()
        cfg.nx = layers
        cfg.precision = 0
        o = ob.Oracle(cfg)
        b = wl.sample_beam(cfg, wl.BeamSpec(16))
        o.load_beam(b)
        o.load_front_plasma(wl.front_plasma(cfg, seed=3))
        t = time.perf_counter()
        o.move_all_split_layers()
        dt = time.perf_counter() - t
        o.close()
        return dt

    t1 = run(2) / 2
    layers = max(2, min(256, int(target_s / max(t1, 1e-3))))
    dt = run(layers)
    np_layer = w.cfg.ny * w.cfg.nz * w.cfg.ppc
    return {"value": np_layer * layers * w.cfg.nx_split / dt, "unit": UNIT, "cores": cores,
            "kind": "port",
            "sample": f"oracle FP64 xi-march of {layers} layers of the {w.cfg.ny}x{w.cfg.nz} "
                      f"grid ({np_layer} particles/layer), {dt:.1f} s on {cores} threads",
            "_seconds": dt}


# ------------------------------------------------------------------ adjoint (c3)
def adjoint_measure(precision: str):
    """The c3 adjoint: 256 x 256 x 2048, 4 ppc, CIC, 1e6-particle driver whose
    charge profile is 64 xi-bins with seeded weights in [0.5, 1.5]; loss = on-axis
    Ex integrated over the witness window xi in [-6, -5] behind the driver
    centre; layer checkpoints every 32 layers.  Reports the forward march and
    the adjoint times (device events), their ratio, the ratio over the same
    layer range (the sweep covers only the layers from the head to the window),
    and the gradient against central differences (h = 1e-3) on a few bins, in
    the same precision and in FP64, and against the FP64 adjoint on all bins."""
    import numpy as np
    import torch
    from tertia_b200 import workload as wl
    from tertia_b200.abi import QS_SHAPE_CIC
    from tertia_b200.autograd import xi_bins
    from tertia_b200.mesh import Mesh

    nbins, every, h = 64, 32, 1e-3

    def setup(prec):
        w = wl.make_workload("c3", prec)
        cfg = w.cfg
        cfg.shape = QS_SHAPE_CIC
        # the beam is deposited where it stands (no beam motion, no
        # radiation loss): the loss is then a function of the bin weights
        # alone, not of the fields an earlier march left for the beam push
        cfg.ts = 0.0
        cfg.synchrotron = 0
        beam = wl.workload_beam(w)
        xc = wl.driver_center_x(cfg, w.beams[0].sigma_xi)
        sx = w.beams[0].sigma_xi
        bins = xi_bins(beam, cfg, nbins, xc - 4 * sx, xc + 4 * sx)
        xl = np.arange(cfg.nx) * cfg.hx
        coeff = np.where((xl >= xc - 6.0) & (xl <= xc - 5.0), cfg.hx, 0.0)
        m = Mesh(cfg)
        m.seed_front_plasma(0)
        m.adjoint_checkpoints(every)
        return cfg, m, beam, bins, coeff

    beta = np.random.default_rng(3).uniform(0.5, 1.5, nbins)

    def forward(m, beam, bins, coeff, b):
        bb = dict(beam)
        bb["w"] = np.asarray(beam["w"]) * b[bins]
        m.load_beam(bb)
        m.move_beam_particles()
        m.move_all_split_layers()
        return float(np.dot(coeff, m.onaxis_ex()))

    def grad(m, beam, bins, coeff, b):
        forward(m, beam, bins, coeff, b)
        dw = m.adjoint(coeff)
        return np.bincount(bins, weights=np.asarray(beam["w"]) * dw, minlength=nbins)

    cfg, m, beam, bins, coeff = setup(precision)
    stream = torch.cuda.ExternalStream(m.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    forward(m, beam, bins, coeff, beta)          # warm-up (captures the march graph)
    g = grad(m, beam, bins, coeff, beta)          # warm-up of the adjoint
    bb = dict(beam)
    bb["w"] = np.asarray(beam["w"]) * beta[bins]
    m.load_beam(bb)
    m.move_beam_particles()
    torch.cuda.synchronize()
    e0.record(stream)
    m.move_all_split_layers()
    e1.record(stream)
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    e0.record(stream)
    dw = m.adjoint(coeff)
    e1.record(stream)
    torch.cuda.synchronize()
    adj_ms = e0.elapsed_time(e1)
    g = np.bincount(bins, weights=np.asarray(beam["w"]) * dw, minlength=nbins)
    lo = int(np.nonzero(coeff)[0].min())
    swept = cfg.nx - lo
    # central differences on the 4 bins with the largest gradient
    top = np.argsort(-np.abs(g))[:4]

    def fd_of(mm):
        out = []
        for b in top:
            bp, bm = beta.copy(), beta.copy()
            bp[b] += h
            bm[b] -= h
            out.append((forward(mm, beam, bins, coeff, bp) - forward(mm, beam, bins, coeff, bm))
                       / (2 * h))
        return np.array(out)

    fd = fd_of(m)
    m.close()
    cfg32, m32, beam32, bins32, coeff32 = setup("fp32")
    g32 = grad(m32, beam32, bins32, coeff32, beta)
    m32.close()
    cfg64, m64, beam64, bins64, coeff64 = setup("fp64")
    g64 = grad(m64, beam64, bins64, coeff64, beta)
    fd64 = fd_of(m64)
    m64.close()
    rel = lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    return {"workload": "c3: 256x256x2048 CIC, 64 xi-bins, witness window xi in [-6, -5], "
                        "beam deposited in place (Ts = 0), "
                        f"checkpoints every {every} layers",
            "precision": precision, "forward_ms": fwd_ms, "adjoint_ms": adj_ms,
            "adjoint_over_forward": adj_ms / fwd_ms,
            "layers_swept": swept, "layers": cfg.nx,
            "adjoint_over_forward_same_layers": adj_ms / (fwd_ms * swept / cfg.nx),
            "grad_rel_err_vs_fd_top4": rel(g[top], fd),
            "grad_rel_err_vs_fp64_fd_top4": rel(g[top], fd64),
            "grad_rel_err_vs_fp64_adjoint": rel(g, g64),
            "fp32_grad_rel_err_vs_fp64_fd_top4": rel(g32[top], fd64),
            "fp32_grad_rel_err_vs_fp64_adjoint": rel(g32, g64),
            "fp64_adjoint_rel_err_vs_fp64_fd_top4": rel(g64[top], fd64),
            "fd_note": "central differences of the loss; in BF16x3 they carry the FP32 rounding "
                       "of the loss divided by 2h, hence the FP64 differences as reference",
            "fd_step": h, "loss_note": "loss = sum over window layers of hx * on-axis Ex",
            "timing": "device events on the handle's stream around the march and around "
                      "qs_adjoint"}


def adjoint_grid_measure(workload="c1", precision="fp32", every=32, nbins=64):
    """The adjoint on the forward's own grid (c1: 512 x 512 x 1024, the
    size the adjoint's cost target is quoted at), with the c3 adjoint's
    loss, bins and checkpoint interval: the driver's charge profile as
    `nbins` xi-bins, loss = on-axis Ex integrated over xi in [-6, -5] behind
    the driver centre, beam deposited in place.  Timing only: the march
    and qs_adjoint (device events on the handle's stream), the third
    of three runs."""
    import numpy as np
    import torch
    from tertia_b200 import workload as wl
    from tertia_b200.abi import QS_SHAPE_CIC
    from tertia_b200.autograd import xi_bins
    from tertia_b200.mesh import Mesh

    w = wl.make_workload(workload, precision)
    cfg = w.cfg
    cfg.shape = QS_SHAPE_CIC
    cfg.ts = 0.0
    cfg.synchrotron = 0
    beam = wl.workload_beam(w)
    xc = wl.driver_center_x(cfg, w.beams[0].sigma_xi)
    sx = w.beams[0].sigma_xi
    bins = xi_bins(beam, cfg, nbins, xc - 4 * sx, xc + 4 * sx)
    xl = np.arange(cfg.nx) * cfg.hx
    coeff = np.where((xl >= xc - 6.0) & (xl <= xc - 5.0), cfg.hx, 0.0)
    beta = np.random.default_rng(3).uniform(0.5, 1.5, nbins)
    bb = dict(beam)
    bb["w"] = np.asarray(beam["w"]) * beta[bins]
    with Mesh(cfg) as m:
        m.seed_front_plasma(0)
        m.adjoint_checkpoints(every)
        st = torch.cuda.ExternalStream(m.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(3):
            m.load_beam(bb)
            m.move_beam_particles()
            torch.cuda.synchronize()
            e0.record(st)
            m.move_all_split_layers()
            e1.record(st)
            torch.cuda.synchronize()
            fwd = e0.elapsed_time(e1)
            e0.record(st)
            m.adjoint(coeff)
            e1.record(st)
            torch.cuda.synchronize()
            adj = e0.elapsed_time(e1)
    lo = int(np.nonzero(coeff)[0].min())
    swept = cfg.nx - lo
    return {"workload": f"{w.name} grid: {cfg.ny}x{cfg.nz}x{cfg.nx} CIC {precision}, the c3 "
                        f"adjoint's loss and {nbins} xi-bins, checkpoints every {every} layers",
            "forward_ms": fwd, "adjoint_ms": adj, "layers_swept": swept, "layers": cfg.nx,
            "adjoint_over_forward_same_layers": adj / (fwd * swept / cfg.nx),
            "timing": "device events on the handle's stream around the checkpointed march and "
                      "around qs_adjoint; third of three runs"}


# ------------------------------------------------------------------ FP64 comparison
STUDY_BITS = (("transforms", 1), ("spectral_state", 2), ("push", 4), ("fields", 8),
              ("beam_currents", 16), ("front_plasma_input", 32), ("particle_state_storage", 64),
              ("push_arithmetic", 128), ("position_storage", 256), ("momentum_storage", 512),
              ("all", 31))


def fp64_compare(cfg, beam, pushes_per_step, ours_ms):
    import numpy as np
    import torch
    from tertia_b200.abi import PRECISIONS
    from tertia_b200.mesh import Mesh

    def run(prec, eps=0.0, study=None):
        c = cfg.copy()
        c.precision = PRECISIONS[prec]
        b = dict(beam)
        if eps:
            b["w"] = np.asarray(beam["w"]) * (1.0 + eps)
        if study is not None:
            os.environ["QS_FP32_STUDY"] = str(study)
        try:
            m = Mesh(c)
        finally:
            os.environ.pop("QS_FP32_STUDY", None)
        m.load_beam(b)
        m.step()                    # identical first step from identical inputs
        stream = torch.cuda.ExternalStream(m.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        m.step()
        e1.record(stream)
        torch.cuda.synchronize()
        out = {"ex": m.onaxis_ex(), "psi": m.psi(), "beam": m.get_beam(),
               "sums": m.charge_sums(), "ms": e0.elapsed_time(e1)}
        m.close()
        return out

    rel = lambda a, b: float(np.linalg.norm(np.asarray(a) - np.asarray(b)) /
                             np.linalg.norm(np.asarray(b)))
    head = slice(3 * cfg.nx // 4, None)    # the head of the box: the highest layers
    r64 = run("fp64")
    r64f = run("fp64fft")
    r32 = run(cfg_precision_name(cfg))

    def errors(r, ref):
        e = {"ez_rel_l2": rel(r["ex"], ref["ex"]),
             "ez_rel_l2_head_quarter": rel(r["ex"][head], ref["ex"][head]),
             "psi_rel_l2": rel(r["psi"], ref["psi"])}
        bo, bm = ref["beam"], r["beam"]
        for k in ("px", "py", "pz"):    # the kicks of the two beam pushes
            e[f"beam_d{k}_rel_l2"] = rel(np.asarray(bm[k]) - np.asarray(beam[k]),
                                         np.asarray(bo[k]) - np.asarray(beam[k]))
        pos = lambda b, c, f: np.asarray(b[c], dtype=np.float64) + np.asarray(b[f])
        e["beam_position_max_abs_cells"] = float(max(
            np.max(np.abs(pos(bm, c, f) - pos(bo, c, f))) for c, f in
            (("i", "x"), ("j", "y"), ("k", "z"))))
        e["beam_cells_equal_fraction"] = float(np.mean(
            (np.asarray(bm["i"]) == np.asarray(bo["i"])) &
            (np.asarray(bm["j"]) == np.asarray(bo["j"])) &
            (np.asarray(bm["k"]) == np.asarray(bo["k"]))))
        for q in ("rho", "jx", "rho_beam"):
            a, b = r["sums"][q], ref["sums"][q]
            e[f"charge_sum_{q}_max_rel"] = float(np.max(np.abs(a - b)) /
                                                 max(np.max(np.abs(b)), 1e-300))
        return e

    e64f = rel(r64f["ex"], r64["ex"])
    e32 = errors(r32, r64)
    out = {"value": pushes_per_step / (r64["ms"] / 1e3), "unit": UNIT,
           "ms_per_step": r64["ms"],
           "speedup": r64["ms"] / ours_ms,
           "transforms": "dense FP64 SIMT matrix passes (O(N^3) per plane)",
           "fft": {"value": pushes_per_step / (r64f["ms"] / 1e3), "unit": UNIT,
                   "ms_per_step": r64f["ms"],
                   "speedup_over_fp64_plain": r64["ms"] / r64f["ms"],
                   "ours_speedup_over_it": r64f["ms"] / ours_ms,
                   "transforms": "FP64 half-length complex FFTs, the FP32 path's algorithm; "
                                 "CIC push grouped by cell as in FP32, FP64 with FMA",
                   "ez_rel_l2_vs_fp64": e64f},
           "errors_vs_fp64": e32,
           "timing": "device events around the second beam step of each run (the same "
                     "inputs; the main line's own timing for ours)"}
    # the fastest path whose whole-box on-axis Ez is within 1e-5 of the plain FP64 path
    cands = [(cfg_precision_name(cfg), ours_ms, e32["ez_rel_l2"]), ("fp64fft", r64f["ms"], e64f)]
    ok = [c for c in cands if c[2] <= 1e-5]
    if ok:
        name, ms, err = min(ok, key=lambda c: c[1])
        out["at_ez_1e-5"] = {"path": name, "value": pushes_per_step / (ms / 1e3), "unit": UNIT,
                             "ms_per_step": ms, "ez_rel_l2_vs_fp64_plain": err,
                             "speedup_over_fp64_plain": r64["ms"] / ms}
    floors = {}
    for tag, eps in (("perturbed_1e-15", 1e-15), ("perturbed_6e-8", 6e-8)):
        floors[tag] = rel(run("fp64", eps)["ex"], r64["ex"])
    out["ez_floor_fp64_vs_itself"] = floors
    att = {}
    for name, bit in STUDY_BITS:
        rs = run("fp64fft", study=bit)
        att[name] = {"ez_rel_l2": rel(rs["ex"], r64f["ex"]),
                     "ez_rel_l2_head_quarter": rel(rs["ex"][head], r64f["ex"][head])}
    out["attribution"] = {
        "base": "fp64fft (FP64 with FFT transforms)", "components": att,
        "note": "each entry: the FP64-FFT march with that part in FP32 (transforms through the "
                "FP32 FFT kernels; spectral state carried between layers rounded to float; the "
                "push through the FP32 push kernel on float particles and fields; the real "
                "field planes rounded to float; the beam currents rounded to float; only the "
                "front plasma's starting state rounded to float; the plasma state rounded to "
                "float after every full push of an FP64 push; the FP32 push kernel's increments "
                "added to an FP64 state), on-axis Ez after two beam steps against the plain "
                "FP64-FFT march"}
    out["ez_note"] = ("on-axis Ex (the reference's longitudinal field) over all layers after 2 "
                      "beam steps; head quarter = the 1/4 of the layers nearest the front")
    return out


def cfg_precision_name(cfg):
    from tertia_b200.abi import PRECISIONS
    inv = {v: k for k, v in PRECISIONS.items()}
    return inv[cfg.precision]


# ------------------------------------------------------------------ c2 precision study
def c2_study(precisions=("fp32", "bf16x3", "tf32x3", "bf16x6"), every=64, shape="cic"):
    """The c2 precision study: 1024 x 1024 x 2048, 4 ppc, n_b/n_0 = 1, 4e6
    driver particles; one beam step in FP64 (FFT transforms) and in each
    FP32 / split-precision mode.  The march runs layer by layer through the
    fine-grained entry points, and at every `every`-th layer the C layer's
    Ex, Ey, Ez, Bx, By, Bz and its corrected density rho are read; per-field
    relative L2 over those layers against FP64.  The beam state stays FP64
    in every mode."""
    import numpy as np
    import torch
    from tertia_b200 import workload as wl
    from tertia_b200.abi import PRECISIONS, QS_SHAPE_CIC, QS_SHAPE_NGP, QS_F_DENS
    from tertia_b200.mesh import Mesh

    w = wl.make_workload("c2")
    cfg = w.cfg
    cfg.shape = QS_SHAPE_CIC if shape == "cic" else QS_SHAPE_NGP
    cfg.use_graph = 0
    beam = wl.workload_beam(w)
    front = None
    names = ["Ex", "Ey", "Ez", "Bx", "By", "Bz", "rho"]
    sample = set(range(cfg.nx - 1, -1, -every))

    head_lo = 3 * cfg.nx // 4     # the head quarter of the box: layers head_lo .. nx-1

    def march(prec, ref=None, eps=0.0, study=None):
        c = cfg.copy()
        c.precision = PRECISIONS[prec]
        if study is not None:
            os.environ["QS_FP32_STUDY"] = str(study)
        try:
            m = Mesh(c)
        finally:
            os.environ.pop("QS_FP32_STUDY", None)
        b = dict(beam)
        if eps:
            b["w"] = np.asarray(beam["w"]) * (1.0 + eps)
        m.load_beam(b)
        m.move_beam_particles()
        m.seed_front_plasma(0)
        m.begin_march()
        got = {}
        num = np.zeros((2, 7))
        den = np.zeros((2, 7))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(cfg.nx - 1, -1, -1):
            m.layer_begin(i, 0)
            m.move_split_layer(i, 0)
            if i in sample:
                planes = [m.get_layer(1, f) for f in range(6)] + [m.get_layer(1, QS_F_DENS)]
                if ref is None:
                    got[i] = planes
                else:
                    for part in (0, 1):
                        if part == 1 and i < head_lo:
                            continue
                        for q in range(7):
                            num[part, q] += float(np.sum((planes[q] - ref[i][q]) ** 2))
                            den[part, q] += float(np.sum(ref[i][q] ** 2))
            m.layer_end(i, 0)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        ex = m.onaxis_ex()
        m.close()
        if ref is None:
            return got, ex, dt
        errs = {part: {n: float(np.sqrt(num[p_, q] / den[p_, q])) for q, n in enumerate(names)}
                for p_, part in enumerate(("whole_box", "head_quarter"))}
        return errs, ex, dt

    ref, ex64, t64 = march("fp64fft")
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    out = {"workload": "c2: 1024x1024x2048, 4 ppc, n_b/n_0 = 1, 4e6 driver particles, "
                       f"{shape.upper()}, one beam step",
           "reference": "FP64 with FFT transforms (QS_PREC_FP64_FFT)",
           "sampled_layers": len(sample), "every": every, "head_quarter_from_layer": head_lo,
           "fields": names, "march_s": {"fp64fft": t64}, "per_field_rel_l2": {},
           "ez_onaxis_rel_l2": {}, "ez_onaxis_rel_l2_head_quarter": {}}
    head = slice(head_lo, None)
    for prec in precisions:
        err, ex, dt = march(prec, ref)
        out["per_field_rel_l2"][prec] = err
        out["ez_onaxis_rel_l2"][prec] = rel(ex, ex64)
        out["ez_onaxis_rel_l2_head_quarter"][prec] = rel(ex[head], ex64[head])
        out["march_s"][prec] = dt
    # floors: FP64 against itself with the beam weights x (1 + 6e-8), and
    # with only the front plasma's starting state rounded to float (what any
    # FP32 representation of the plasma starts from)
    floors = {}
    for tag, kw in (("fp64_beam_weights_x(1+6e-8)", {"eps": 6e-8}),
                    ("fp64_front_plasma_rounded_to_float", {"study": 32})):
        err, ex, _ = march("fp64fft", ref, **kw)
        floors[tag] = {"per_field_rel_l2": err, "ez_onaxis_rel_l2": rel(ex, ex64),
                       "ez_onaxis_rel_l2_head_quarter": rel(ex[head], ex64[head])}
    out["floors"] = floors
    out["timing"] = ("host clock around the layer-by-layer march (eager launches and the plane "
                     "reads of the sampled layers included): for scale only")
    return out


# ------------------------------------------------------------------ c4 full form
def c4_measure(precision="fp32", shape="cic", fp64_head_layers=1024, nbins=64, every=64):
    """The c4 full form on one GPU: 1024 x 1024 x 4096, 4 ppc with thermal
    spread 0.01, a 1e7-particle bi-Gaussian driver plus a 1e6-particle
    witness (sigma_r 0.3, sigma_xi 0.3) at xi = -5.5.

    - memory: device bytes the handle holds (forward, then with the layer
      checkpoints every `every` layers and the adjoint's buffers), against
      the GPU's total;
    - forward: one beam step (beam push + march) timed with device events
      after an untimed one;
    - adjoint: the driver's charge profile as `nbins` xi-bins, loss = on-axis
      Ex integrated over the witness window xi in [-6, -5] behind the driver
      centre, checkpoints every `every` layers; the adjoint timed against the
      march over the same layers (device events around both);
    - error against FP64: the full FP64 field store of c4 (201 GB) exceeds one
      GPU, so FP64 (FFT transforms) runs the head `fp64_head_layers` layers
      with the beam particles in them, and the first step's on-axis Ex of
      those layers is compared (the march runs from the head, so they do not
      depend on the layers behind them)."""
    import numpy as np
    import torch
    from tertia_b200 import workload as wl
    from tertia_b200.abi import PRECISIONS, QS_SHAPE_CIC, QS_SHAPE_NGP
    from tertia_b200.autograd import xi_bins
    from tertia_b200.mesh import Mesh

    w = wl.make_workload("c4", precision)
    cfg = w.cfg
    cfg.shape = QS_SHAPE_CIC if shape == "cic" else QS_SHAPE_NGP
    beam = wl.workload_beam(w)
    nb = len(beam["x"])
    npl = cfg.ny * cfg.nz * cfg.ppc
    free0, total = torch.cuda.mem_get_info()
    out = {"workload": f"{w.name}: {w.description}, {shape.upper()}, {precision}",
           "beam_particles": nb, "plasma_particles_per_layer": npl}

    def events(m):
        st = torch.cuda.ExternalStream(m.stream())
        return st, torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    m = Mesh(cfg)
    m.load_beam(beam)
    m.step()                                   # untimed: the march graph is captured
    ex_first = m.onaxis_ex()
    st, e0, e1 = events(m)
    torch.cuda.synchronize()
    e0.record(st)
    m.step()
    e1.record(st)
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    used_fwd = free0 - torch.cuda.mem_get_info()[0]
    out["forward"] = {"ms_per_step": fwd_ms,
                      "value": npl * cfg.nx * cfg.nx_split / (fwd_ms / 1e3), "unit": UNIT,
                      "timing": "device events around one beam step (beam push + march)"}
    # the adjoint on the first step's beam (deposited in place, Ts = 0)
    m.close()
    c = cfg.copy()
    c.ts = 0.0
    c.synchrotron = 0
    m = Mesh(c)
    xc = wl.driver_center_x(c, w.beams[0].sigma_xi)
    sx = w.beams[0].sigma_xi
    drv = np.arange(nb) < w.beams[0].n
    bins = xi_bins(beam, c, nbins, xc - 4 * sx, xc + 4 * sx)
    beta = np.random.default_rng(3).uniform(0.5, 1.5, nbins)
    bw = dict(beam)
    bw["w"] = np.where(drv, np.asarray(beam["w"]) * beta[bins], beam["w"])
    xl = np.arange(c.nx) * c.hx
    coeff = np.where((xl >= xc - 6.0) & (xl <= xc - 5.0), c.hx, 0.0)
    m.seed_front_plasma(0)
    m.adjoint_checkpoints(every)
    m.load_beam(bw)
    m.move_beam_particles()
    m.move_all_split_layers()                  # capture
    m.adjoint(coeff)                           # capture of the sweep
    m.seed_front_plasma(0)
    m.move_all_split_layers()
    st, e0, e1 = events(m)
    torch.cuda.synchronize()
    e0.record(st)
    m.move_all_split_layers()
    e1.record(st)
    torch.cuda.synchronize()
    march_ms = e0.elapsed_time(e1)
    e0.record(st)
    dw = m.adjoint(coeff)
    e1.record(st)
    torch.cuda.synchronize()
    adj_ms = e0.elapsed_time(e1)
    used_adj = free0 - torch.cuda.mem_get_info()[0]
    lo = int(np.nonzero(coeff)[0].min())
    swept = c.nx - lo
    g = np.bincount(bins[drv], weights=(np.asarray(beam["w"]) * dw)[drv], minlength=nbins)
    out["adjoint"] = {"checkpoint_every": every, "bins": nbins, "march_ms": march_ms,
                      "adjoint_ms": adj_ms, "layers_swept": swept, "layers": c.nx,
                      "adjoint_over_forward_same_layers": adj_ms / (march_ms * swept / c.nx),
                      "adjoint_over_forward": adj_ms / march_ms,
                      "grad_norm": float(np.linalg.norm(g)),
                      "timing": "device events on the handle's stream around the march and "
                                "around qs_adjoint"}
    m.close()
    out["memory"] = {"device_bytes_forward": int(used_fwd),
                     "device_bytes_with_adjoint": int(used_adj),
                     "gpu_total_bytes": int(total),
                     "fraction_of_gpu": used_adj / total,
                     "layout": "field store (nx+1) x 6 planes, beam currents (nx+1) x 2 planes "
                               "(their spectra computed in place), layer checkpoints, the "
                               "adjoint's beam-spectrum adjoint only for the swept layers"}
    # FP64 over the head layers
    hl = min(fp64_head_layers, cfg.nx)
    keep = np.asarray(beam["i"]) >= cfg.nx - hl
    hb = {k: np.ascontiguousarray(np.asarray(v)[keep]) for k, v in beam.items()}
    hb["i"] = (hb["i"] - (cfg.nx - hl)).astype(np.int32)
    res = {}
    for prec in ("fp64fft", precision):
        ch = cfg.copy()
        ch.nx = hl
        ch.precision = PRECISIONS[prec]
        mh = Mesh(ch)
        mh.load_beam(hb)
        mh.step()
        res[prec] = mh.onaxis_ex()
        mh.close()
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    out["error_vs_fp64"] = {
        "layers": f"the head {hl} layers (FP64 store of the whole box exceeds one GPU)",
        "ez_rel_l2_full_box_run": rel(ex_first[cfg.nx - hl + 1:], res["fp64fft"][1:]),
        "ez_rel_l2_same_head_box": rel(res[precision][1:], res["fp64fft"][1:]),
        "note": "first beam step, on-axis Ex of the head layers but the last (whose beam "
                "currents in the head box lack the deposits of the particles behind it); "
                "full_box_run = the c4 run's own head layers, same_head_box = the same "
                "precision on the head box"}
    return out


# ------------------------------------------------------------------ our arm
def next_rows_measure(cfg, beam, uniform_ms, pushes_per_step, steps=2):
    """The rows beside the march, on the bench's own workload and beam:

    - a march through a non-uniform plasma (a Gaussian channel whose density
      ramps along xi; the device seeding weights every cell by the profile and
      the maps read the density at the head each layer), timed like the main
      line (device events on the handle's stream, one warm-up step);
    - the xi-pipeline hand-off: PackLayer of the tail layer with the plasma in
      flight into a pinned host buffer and UnpackLayer of it, by the host
      clock around the synchronous calls, and a march that starts from the
      received layer (device events)."""
    import numpy as np
    import torch
    from tertia_b200 import abi
    from tertia_b200.mesh import Mesh

    def timed_steps(m, n):
        stream = torch.cuda.ExternalStream(m.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(n):
            m.step()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    out = {}
    xf = cfg.hx * cfg.nx
    prof = abi.density_profile(distribution=abi.DIST_GAUSS_CHANNEL, density=0.5, density1=1.5,
                               delta=0.6, radius=0.4, begin=0.0, plateau_begin=0.0,
                               plateau_end=xf + 4.0, end=1e9)
    with Mesh(cfg) as m:
        m.set_density_profile(prof)
        m.load_beam(beam)
        m.step()
        ms = timed_steps(m, steps)
        out["density_profile"] = {
            "profile": "Gaussian channel (density 0.5 on axis, 1.5 outside, radius 0.4) "
                       "ramping up along xi over the box (DIST_GAUSS_CHANNEL)",
            "steps": steps, "ms_per_step": ms, "value": pushes_per_step / (ms / 1e3),
            "unit": UNIT, "over_uniform_ms": ms / uniform_ms,
            "onaxis_ex_max": float(np.abs(m.onaxis_ex()).max())}
    with Mesh(cfg) as m:
        m.load_beam(beam)
        m.step()
        n = m.pack_size()
        buf = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
        reps = 3
        m.pack_layer(out=buf)            # one untimed call each: the device buffers are made
        m.unpack_layer(buf)
        m.sync()
        t0 = time.perf_counter()
        for _ in range(reps):
            m.pack_layer(out=buf)
        t_pack = (time.perf_counter() - t0) / reps
        t0 = time.perf_counter()
        for _ in range(reps):
            m.unpack_layer(buf)
        t_unpack = (time.perf_counter() - t0) / reps
        m.step()                         # from the received layer: the march is rebuilt
        m.unpack_layer(buf)
        ms_recv = timed_steps(m, 1)
        nbytes = n * 8
        out["handoff"] = {
            "buffer_bytes": nbytes, "layout": "12 planes + 12 x Np particle values (doubles)",
            "pack_ms": t_pack * 1e3, "unpack_ms": t_unpack * 1e3,
            "pack_gbs": nbytes / t_pack / 1e9, "unpack_gbs": nbytes / t_unpack / 1e9,
            "march_from_received_layer_ms": ms_recv,
            "over_uniform_ms": ms_recv / uniform_ms}
    return out


def run_ours(args):
    import numpy as np
    import torch
    from tertia_b200 import workload as wl
    from tertia_b200.abi import PRECISIONS, QS_SHAPE_CIC, QS_SHAPE_NGP
    from tertia_b200.mesh import Mesh

    from tertia_b200 import replicas
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    replicas.init(world, local, "nccl", timeout_s=300)
    w = wl.make_workload(args.workload, args.precision)
    cfg = w.cfg
    cfg.shape = QS_SHAPE_CIC if args.shape == "cic" else QS_SHAPE_NGP
    cfg.device = local
    cfg.seed = 12345 + rank
    if args.layers:
        cfg.nx = args.layers
        w.name = f"{w.name}-L{args.layers}"
        w.description = (f"profiling case: {cfg.ny}x{cfg.nz} grid of {args.workload}, "
                         f"{args.layers} layers, 1e5-particle beam at n_b/n_0 = 1e-4")
        beam = wl.sample_beam(cfg, wl.BeamSpec(100_000, nb_over_n0=1e-4))
    else:
        beam = wl.workload_beam(w)
    npl = cfg.ny * cfg.nz * cfg.ppc
    pushes_per_step = npl * cfg.nx * cfg.nx_split

    def barrier():
        replicas.barrier(world)

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, world, "cuda")

    m = Mesh(cfg)
    m.load_beam(beam)
    stream = torch.cuda.ExternalStream(m.stream())
    for _ in range(args.warmup):
        m.step()
    # ---------------- timed region: K steps, device events on the handle's stream
    clocks = ClockSampler(local)
    clocks.start()
    l0 = m.kernel_launches()
    barrier()
    torch.cuda.synchronize()
    clocks.mark()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        m.step()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    clk = clocks.stop()
    launches = m.kernel_launches() - l0
    ms_max = max_over_ranks(ms)
    value = replicas.whole_job_rate(pushes_per_step, world, ms_max)
    onaxis = m.onaxis_ex()

    # ---------------- e2e: the public C ABI with host buffers (pinned)
    n = len(beam["x"])
    pin = {}
    for k in ("i", "j", "k"):
        t = torch.empty(n, dtype=torch.int32, pin_memory=True)
        t.numpy()[:] = beam[k]
        pin[k] = t
    for k in ("x", "y", "z", "px", "py", "pz", "w"):
        t = torch.empty(n, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = beam[k]
        pin[k] = t
    host = {k: v.numpy() for k, v in pin.items()}
    out_pin = {k: torch.empty(n, dtype=torch.int32 if k in "ijk" else torch.float64,
                              pin_memory=True).numpy() for k in ("i", "j", "k", "x", "y", "z",
                                                                 "px", "py", "pz")}
    e2e_steps = max(1, args.steps)
    m.step_host(host, out=out_pin)           # warm the host path
    barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(e2e_steps):
        res, ex = m.step_host(host, out=out_pin)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1) / e2e_steps)
    h2d = n * (3 * 4 + 7 * 8)
    d2h = n * (3 * 4 + 6 * 8) + cfg.nx * 8

    # ---------------- per-class kernel time over one more step: eager launches,
    # an event pair around every launch (host launch gaps are included, so
    # short kernels read long; the shares are cross-checked with ncu)
    m.profile_enable(True)
    torch.cuda.synchronize()
    m.step()
    prof = m.profile_read()
    m.profile_enable(False)

    # ---------------- the dominant kernel timed back to back: the inverse E,B
    # transform pass of the march (6 planes, one y- or z-pass per launch),
    # repeated with the launches queued ahead of the GPU
    gemm = None
    fftp = None
    # the CIC push (the dominant kernel of the FP32 march): the half push and
    # the full push of the head layer, each repeated through the fine-grained
    # entry points with every launch bracketed by events on the handle's
    # stream (one push per call; the full push stores the particles, and every
    # second one is followed by the regrouping, timed apart)
    pushk = None
    if cfg.shape == QS_SHAPE_CIC:
        m.load_front_plasma(wl.front_plasma(cfg, seed=5))
        m.begin_march()
        m.layer_begin(cfg.nx - 1, 0)
        m.guess_fields(cfg.nx - 1, 0)
        pushk = {"particles": cfg.ny * cfg.nz * cfg.ppc}
        for kind, full in (("half", 0), ("full", 1)):
            for _ in range(3):
                m.move_particles_layer(cfg.nx - 1, 0, full)
            m.sync()
            m.profile_enable(True)
            for _ in range(40):
                m.move_particles_layer(cfg.nx - 1, 0, full)
            pp = m.profile_read()
            m.profile_enable(False)
            p_ms, p_n = pp["push_deposit"]
            pushk[kind] = {"launches": p_n, "avg_launch_us": p_ms * 1e3 / max(p_n, 1)}
        pushk["avg_launch_us"] = 0.5 * (pushk["half"]["avg_launch_us"] +
                                        pushk["full"]["avg_launch_us"])
    if args.precision == "fp32":
        # FFT passes (power-of-two grids): 2 launches per transform, each
        # reading and writing the 6 planes once
        nf = 6
        xs = torch.randn(nf, cfg.nz, cfg.ny, device="cuda", dtype=torch.float32)
        ys = torch.empty_like(xs)
        for _ in range(3):
            m.transform2d_dev(0, 1, nf, xs.data_ptr(), ys.data_ptr())
        m.sync()
        reps = 200
        ev0.record(stream)
        for _ in range(reps):
            m.transform2d_dev(0, 1, nf, xs.data_ptr(), ys.data_ptr())
        ev1.record(stream)
        m.sync()
        loop_us = ev0.elapsed_time(ev1) * 1e3 / reps
        fftp = {"planes": nf, "launches_per_transform": 2, "avg_launch_us": loop_us / 2.0,
                "loop_us_per_transform": loop_us}
        del xs, ys
    if args.precision in ("bf16x3", "tf32x3", "bf16x6"):
        nf = 6
        xs = torch.randn(nf, cfg.nz, cfg.ny, device="cuda", dtype=torch.float32)
        ys = torch.empty_like(xs)
        for _ in range(3):
            m.transform2d_dev(0, 1, nf, xs.data_ptr(), ys.data_ptr())
        m.sync()
        reps = 200
        ev0.record(stream)
        for _ in range(reps):
            m.transform2d_dev(0, 1, nf, xs.data_ptr(), ys.data_ptr())
        ev1.record(stream)
        m.sync()
        loop_ms = ev0.elapsed_time(ev1)
        m.profile_enable(True)
        for _ in range(reps):
            m.transform2d_dev(0, 1, nf, xs.data_ptr(), ys.data_ptr())
        m.sync()
        p2 = m.profile_read()
        m.profile_enable(False)
        g_ms, g_n = p2["transform_gemm"]
        s_ms, _ = p2["transform_split"]
        # the back-to-back loop (no events between launches) gives the time of
        # one transform = split + 2 passes; the evented run gives the passes'
        # share of it (its per-launch times include launch gaps)
        share = g_ms / max(g_ms + s_ms, 1e-12)
        loop_us = loop_ms * 1e3 / reps
        gemm = {"planes": nf, "launches_per_transform": 2,
                "avg_launch_us": loop_us * share / 2.0,
                "loop_us_per_transform": loop_us, "pass_share_evented": share,
                "evented_avg_launch_us": g_ms * 1e3 / max(g_n, 1)}
        del xs, ys
    m.close()

    # ---------------- FP64 paths on the same inputs: speed and the errors.
    # Two beam steps each (the second step's beam push sees the first march's
    # fields); the second step is timed with device events.
    #  - fp64: the plain FP64 path with dense-matrix transforms (the
    #    denominator of the >= 5x target); fp64fft: FP64 with the same FFT
    #    algorithm as the FP32 path (separates algorithm from precision);
    #  - the FP32 path's errors against fp64: on-axis Ez (the reference's Ex)
    #    over the whole box and its head quarter, psi, the beam phase space,
    #    the FP64 charge sums;
    #  - floors: fp64 against itself with the beam weights x (1 + eps);
    #  - attribution: the FP64-FFT path with one part of the march in FP32
    #    at a time (QS_FP32_STUDY), against the plain FP64-FFT path.
    fp64 = None
    if not args.no_fp64:
        fp64 = fp64_compare(cfg, beam, pushes_per_step, ms)

    # ---------------- roofline of the dominant kernel
    hbm, bf16, bf16_sus, src = peaks()
    dom = max(prof, key=lambda k: prof[k][0])
    L, N, S, nit = cfg.nx, cfg.ny, cfg.nx_split, cfg.n_iter
    if gemm:
        # one launch = one K = N pass over 6 N x N planes: 6 * 2 N^3 algorithmic
        # flops (the split products, 3x or 6x that, are executed work)
        flops_launch = gemm["planes"] * 2.0 * cfg.ny * cfg.nz * cfg.ny
        achieved = flops_launch / (gemm["avg_launch_us"] / 1e6) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": bf16, "unit": "TFLOP/s",
                "frac": achieved / bf16, "peak_source": f"bf16_tflops (burst) of {src}",
                "kernel": "dtt_tc_kernel (transform pass, 6 planes)",
                "flops_per_launch": flops_launch, "avg_launch_us": gemm["avg_launch_us"],
                "executed_flop_multiplier": {"bf16x3": 3, "tf32x3": 3, "bf16x6": 6}[
                    args.precision],
                "timing": gemm}
        # transforms per (layer, split) in the march: 6 (Guess inverse E, B)
        # + (nIter+1) * (3 forward J + 6 inverse E, B) + 2 beam planes
        roof["march_transforms_per_layer"] = 6 + (nit + 1) * 9 + 2
    elif pushk:
        # a layer pushes every plasma particle twice (nIter = 1): the half push
        # reads 28 B of particle state plus the P and C fields (12 values) and
        # the deposit (4 values) of its cell shared by the ppc particles, 4 B
        # each; the full push also writes the 24 B of state.  112 B per
        # particle-layer push over the two launches, 56 B per launch on average
        b_half = 28.0 + 16.0 * 4.0 / cfg.ppc
        b_full = b_half + 24.0
        bpp = 0.5 * (b_half + b_full)
        bytes_launch = bpp * pushk["particles"]
        achieved = bytes_launch / (pushk["avg_launch_us"] / 1e6) / 1e9
        for kind, b in (("half", b_half), ("full", b_full)):
            pushk[kind]["bytes_per_particle"] = b
            pushk[kind]["achieved_gbs"] = (b * pushk["particles"] /
                                           (pushk[kind]["avg_launch_us"] / 1e6) / 1e9)
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": f"hbm_gbs of {src}",
                "kernel": "push_cic_row_kernel (CIC push + deposit; the half and the full push "
                          "of a layer, averaged per launch)",
                "bytes_per_particle": bpp, "bytes_per_launch": bytes_launch,
                "avg_launch_us": pushk["avg_launch_us"], "timing": pushk}
        if fftp:
            # the transform pass, for reference: 6 N x N planes read and written
            tb = fftp["planes"] * 2.0 * 4.0 * cfg.ny * cfg.nz
            roof["transform_pass"] = {
                "kernel": "fft_rows_kernel / fft_cols_kernel (6 planes)", "bytes_per_launch": tb,
                "avg_launch_us": fftp["avg_launch_us"],
                "achieved_gbs": tb / (fftp["avg_launch_us"] / 1e6) / 1e9, "timing": fftp}
    else:
        roof = {"bound": "hbm", "achieved": None, "peak": hbm, "unit": "GB/s", "frac": None,
                "kernel": dom}
    tr = traffic_record("dtt_tc_kernel" if gemm else ("push_cic_row_kernel" if pushk else dom),
                        args.workload, args.precision)
    roof["traffic"] = tr.get("bytes_per_launch") if tr else None
    if tr:
        roof["traffic_source"] = tr.get("source")
    roof["evented_kernel_ms_per_step"] = {k: round(v[0], 3) for k, v in prof.items()}
    roof["kernel_launches_per_step"] = {k: v[1] for k, v in prof.items()}
    roof["dominant_class_evented"] = dom

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(w, args.cpu_seconds)
        cpu.pop("_seconds")
    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint and not args.layers:
        adjoint = adjoint_measure(args.precision)
        # the same adjoint on the forward's grid (a failure is reported, not fatal)
        try:
            adjoint["on_forward_grid"] = adjoint_grid_measure(args.workload, args.precision)
        except Exception as e:   # noqa: BLE001
            adjoint["on_forward_grid"] = {"error": f"{type(e).__name__}: {e}"}
    nxt = None
    if rank == 0 and world == 1 and not args.no_next and not args.layers:
        # auxiliary rows: a failure here is reported in the line, not fatal to it
        try:
            nxt = next_rows_measure(cfg, beam, ms_max, pushes_per_step)
        except Exception as e:   # noqa: BLE001
            nxt = {"error": f"{type(e).__name__}: {e}"}

    c2 = None
    if rank == 0 and world == 1 and not args.no_c2 and not args.layers:
        try:
            c2 = c2_study(shape=args.shape)
        except Exception as e:   # noqa: BLE001
            c2 = {"error": f"{type(e).__name__}: {e}"}
    c4 = None
    if rank == 0 and world == 1 and not args.no_c4 and not args.layers:
        try:
            c4 = c4_measure(precision=args.precision, shape=args.shape)
        except Exception as e:   # noqa: BLE001
            c4 = {"error": f"{type(e).__name__}: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{w.name}: {w.description}", "ny": cfg.ny, "nz": cfg.nz,
                       "layers": cfg.nx, "ppc": cfg.ppc, "plasma_particles_per_layer": npl,
                       "beam_particles": n, "n_iter": cfg.n_iter, "nx_split": cfg.nx_split,
                       "precision": args.precision, "shape": args.shape,
                       "step": "one beam step: beam push + full xi-march",
                       "l2": "inputs larger than L2 (field store 6.4 GB, beam currents 2.1 GB)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": replicas.whole_job_rate(pushes_per_step, world, e2e_ms),
                    "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_ms},
            "gpu_launches": launches,
            "roofline": roof,
            "cpu_baseline": cpu,
            "fp64_plain": fp64,
            "adjoint": adjoint,
            "next_rows": nxt,
            "c2_precision_study": c2,
            "c4": c4,
            "clocks": clk,
            "onaxis_ex_max": float(np.max(np.abs(onaxis))),
        }
        print(json.dumps(line), flush=True)
    replicas.finish(world)


# ------------------------------------------------------------ reference arm
def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from tertia_b200 import workload as wl
    from tertia_b200.abi import QS_SHAPE_CIC, QS_SHAPE_NGP
    w = wl.make_workload(args.workload)
    w.cfg.shape = QS_SHAPE_CIC if args.shape == "cic" else QS_SHAPE_NGP
    per_step = max(1.0, min(6.0, 150.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_sample(w, per_step)
    vals, secs = [], []
    last = None
    for _ in range(args.steps):
        last = cpu_sample(w, per_step)
        vals.append(last["value"])
        secs.append(last.pop("_seconds"))
    value = statistics.median(vals)
    cpu = dict(last)
    cpu["value"] = value
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": statistics.median(secs) * 1e3,
        "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": f"{w.name}: {w.description}", "ny": w.cfg.ny, "nz": w.cfg.nz,
                   "layers": w.cfg.nx, "ppc": w.cfg.ppc, "shape": args.shape,
                   "sampled": "each step is a bounded sample of this workload: the oracle's "
                              "xi-march over a few layers of its full transverse grid (the "
                              "per-layer cost does not depend on the beam); ms_per_step is the "
                              "sample's own time, value its pushes/s",
                   "parallelism": "host threads"},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference cannot be built here (needs FFTW3, HDF5, MPI); this times the "
                "oracle's C++ restatement of its FP64 host path",
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
