"""Device timeline of the march, from the traced library (libqsb200_trace.so).

    python -m tertia_b200.trace [--workload c1] [--precision fp32] [--grid N]
                                [--layers L] [--warmup 3] [--records 2097152]
                                [--keep 524288] [--out PREFIX] [--onaxis FILE]

Runs `warmup` beam steps of the workload (the first captures the march
graph) and one step timed with device events, attaches a ring of records
(include/qsb200_trace.h), runs one more step, then reads the newest `keep`
records back and prints:

- per kernel kind and grid: the launches seen whole, the mean and median
  span from the first CTA whose dependency wait returned to the last CTA's
  end, and the mean time between the first CTA's start and that return (how
  early the launch was scheduled beside its predecessor);
- the period between successive half pushes (one layer of the march), over
  the layers with and without a plasma regrouping.

The two timed steps show the stamps' own cost.  The records go to
PREFIX_rec.npy; --onaxis saves the on-axis Ex after the traced step.
"""
from __future__ import annotations

import argparse

import numpy as np

KIND_NAMES = {1: "push (no stores)", 2: "push (stores)", 3: "z-pass", 4: "y-pass",
              5: "map: predictor", 6: "map: corrector", 8: "map: corrector + next predictor",
              10: "regroup: offsets", 11: "regroup: scatter"}


def decode(rec: np.ndarray) -> dict:
    """Fields of the ring's records (rows of 4 uint64); empty slots dropped."""
    rec = np.asarray(rec).astype(np.uint64).reshape(-1, 4)
    rec = rec[rec[:, 0] > 0]
    meta = rec[:, 3]
    return {"t0": rec[:, 0].astype(np.int64), "t1": rec[:, 1].astype(np.int64),
            "t2": rec[:, 2].astype(np.int64),
            "kind": (meta >> np.uint64(56)).astype(np.int64),
            "gy": ((meta >> np.uint64(48)) & np.uint64(0xff)).astype(np.int64),
            "by": ((meta >> np.uint64(40)) & np.uint64(0xff)).astype(np.int64),
            "sm": ((meta >> np.uint64(32)) & np.uint64(0xff)).astype(np.int64),
            "bx": (meta & np.uint64(0xffffffff)).astype(np.int64)}


def launches(d: dict) -> list[dict]:
    """Group the records into launches: in order of CTA start, a record opens
    a new launch of its (kind, grid y) when its block index was already seen
    in the open one.  Concurrent launches of the same kind and grid (the two
    z-passes at a layer's end) can mix; `complete` marks the launches with
    the kind's usual number of CTAs."""
    order = np.argsort(d["t0"], kind="stable")
    open_: dict = {}
    out: list[dict] = []
    for i in order:
        key = (int(d["kind"][i]), int(d["gy"][i]))
        blk = (int(d["bx"][i]), int(d["by"][i]))
        L = open_.get(key)
        if L is None or blk in L["seen"]:
            L = {"kind": key[0], "gy": key[1], "seen": set(), "idx": []}
            open_[key] = L
            out.append(L)
        L["seen"].add(blk)
        L["idx"].append(i)
    res = []
    for L in out:
        ii = np.array(L["idx"])
        res.append({"kind": L["kind"], "gy": L["gy"], "ctas": len(ii),
                    "entry": int(d["t0"][ii].min()), "wait": int(d["t1"][ii].min()),
                    "last_wait": int(d["t1"][ii].max()), "end": int(d["t2"][ii].max())})
    res.sort(key=lambda r: r["wait"])
    usual: dict = {}
    for r in res:
        usual.setdefault((r["kind"], r["gy"]), []).append(r["ctas"])
    for r in res:
        r["complete"] = r["ctas"] == max(usual[(r["kind"], r["gy"])])
    return res


def kind_table(ls: list[dict], skip: int = 0) -> list[dict]:
    """Per (kind, grid y): whole launches, mean and median span (us), mean
    wait of the first CTA (us); the first `skip` launches (cut by the ring's
    start) are left out."""
    rows: dict = {}
    for r in ls[skip:]:
        if not r["complete"]:
            continue
        rows.setdefault((r["kind"], r["gy"], r["ctas"]), []).append(r)
    out = []
    for (k, gy, n), v in sorted(rows.items()):
        span = np.array([x["end"] - x["wait"] for x in v]) / 1e3
        pre = np.array([x["wait"] - x["entry"] for x in v]) / 1e3
        out.append({"kind": k, "name": KIND_NAMES.get(k, str(k)), "gy": gy, "ctas": n,
                    "launches": len(v), "span_mean_us": float(span.mean()),
                    "span_median_us": float(np.median(span)), "first_wait_us": float(pre.mean())})
    return out


def layer_periods(ls: list[dict]) -> dict:
    """Periods between successive half pushes (the first CTA past its wait),
    split by whether a regrouping scatter started within the period."""
    halves = [r["wait"] for r in ls if r["kind"] == 1 and r["complete"]]
    scat = np.array([r["wait"] for r in ls if r["kind"] == 11])
    per, reg = [], []
    for a, b in zip(halves[:-1], halves[1:]):
        per.append((b - a) / 1e3)
        reg.append(bool(((scat >= a) & (scat < b)).any()) if scat.size else False)
    per, reg = np.array(per), np.array(reg, dtype=bool)

    def mean(x):
        return float(x.mean()) if x.size else float("nan")

    return {"layers": int(per.size), "mean_us": mean(per), "regroup_us": mean(per[reg]),
            "regroup_layers": int(reg.sum()), "plain_us": mean(per[~reg]),
            "plain_layers": int((~reg).sum())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c1")
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--grid", type=int, default=0)
    ap.add_argument("--layers", type=int, default=0)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--records", type=int, default=1 << 21)
    ap.add_argument("--keep", type=int, default=1 << 19)
    ap.add_argument("--out", default="")
    ap.add_argument("--onaxis", default="")
    args = ap.parse_args()

    from . import abi
    abi.use_trace_library()
    import ctypes as C

    import torch

    from . import workload as wl
    from .abi import QS_SHAPE_CIC
    from .mesh import Mesh

    L = abi.load_library()
    L.qs_trace_attach.argtypes = [C.c_void_p, C.c_void_p, C.c_uint]
    L.qs_trace_attach.restype = C.c_int
    w = wl.make_workload(args.workload, args.precision)
    cfg = w.cfg
    cfg.shape = QS_SHAPE_CIC
    if args.grid:
        cfg.ny = cfg.nz = args.grid
    if args.layers:
        cfg.nx = args.layers
    if args.grid or args.layers:
        beam = wl.sample_beam(cfg, wl.BeamSpec(100_000, nb_over_n0=1e-4))
    else:
        beam = wl.workload_beam(w)
    nrec = args.records
    if nrec <= 0 or nrec & (nrec - 1):
        raise SystemExit("--records must be a power of two")
    keep = min(args.keep, nrec)
    ring = torch.zeros(4 * nrec, dtype=torch.int64, device="cuda")
    pos = torch.zeros(1, dtype=torch.int32, device="cuda")
    with Mesh(cfg) as m:
        m.load_beam(beam)
        st = torch.cuda.ExternalStream(m.stream())
        for _ in range(args.warmup):
            m.step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        m.step()
        e1.record(st)
        torch.cuda.synchronize()
        ms_plain = e0.elapsed_time(e1)
        if L.qs_trace_attach(ring.data_ptr(), pos.data_ptr(), nrec) != 0:
            raise RuntimeError("qs_trace_attach failed")
        try:
            e0.record(st)
            m.step()
            e1.record(st)
            torch.cuda.synchronize()
        finally:
            L.qs_trace_attach(None, None, 0)
        ms_traced = e0.elapsed_time(e1)
        if args.onaxis:
            np.save(args.onaxis, m.onaxis_ex())
    n = int(pos.item()) & 0xffffffff
    rec = ring.cpu().numpy().reshape(-1, 4)
    # the newest `keep` records, oldest first
    idx = (np.arange(n - keep, n) % nrec) if n > nrec else np.arange(max(0, n - keep), n)
    rec = rec[idx]
    if args.out:
        np.save(args.out + "_rec.npy", rec)
    d = decode(rec)
    ls = launches(d)
    print(f"trace: {cfg.ny}x{cfg.nz}x{cfg.nx} {args.precision}, one beam step "
          f"{ms_plain:.2f} ms untraced, {ms_traced:.2f} ms traced; {n} records, "
          f"the newest {len(d['t0'])} read")
    print(f"{'kernel':>32} {'grid y':>6} {'CTAs':>5} {'launches':>8} {'span mean':>9} "
          f"{'median':>7} {'first wait':>10}  (us)")
    for r in kind_table(ls, skip=8):
        print(f"{r['name']:>32} {r['gy']:>6} {r['ctas']:>5} {r['launches']:>8} "
              f"{r['span_mean_us']:>9.2f} {r['span_median_us']:>7.2f} {r['first_wait_us']:>10.2f}")
    p = layer_periods(ls)
    print(f"layer period (half push to half push): {p['mean_us']:.2f} us over {p['layers']} "
          f"layers; with a regrouping {p['regroup_us']:.2f} us ({p['regroup_layers']}), "
          f"without {p['plain_us']:.2f} us ({p['plain_layers']})")


if __name__ == "__main__":
    main()
