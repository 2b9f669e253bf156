"""The device timeline's host side (tertia_b200/trace.py) on a synthetic ring,
and the traced library's exports (no GPU needed)."""
import ctypes as C
import os

import numpy as np
import pytest

from test_abi import ROOT, header_functions
from tertia_b200 import trace as tr


def _rec(kind, t0, t1, t2, bx, by=0, gy=1, sm=0):
    meta = (kind << 56) | (gy << 48) | (by << 40) | (sm << 32) | bx
    return [t0, t1, t2, meta]


def _layer(t, regroup):
    """One layer of the march, 4 CTAs per launch (x 6 or 3 planes for the
    z-passes), times in ns from t."""
    recs, at = [], t
    seq = [(1, 1, 30000), (3, 3, 4000), (6, 1, 8000), (3, 6, 5000), (2, 1, 30000),
           (3, 3, 4000), (8, 1, 14000), (3, 6, 5000)]
    for kind, gy, dur in seq:
        for b in range(4):
            for y in range(gy):
                recs.append(_rec(kind, at - 500, at + 10 * b, at + dur - 10 * b, b, y, gy))
        if kind == 2 and regroup:   # the scatter beside what follows the full push
            for b in range(4):
                recs.append(_rec(11, at + dur + 100, at + dur + 200, at + dur + 9000, b))
        at += dur + 1000
    return recs, at


def test_launches_and_layer_periods():
    recs, t, periods = [], 10_000_000, []
    for layer in range(5):
        r, t2 = _layer(t, regroup=layer % 2 == 1)
        recs += r
        periods.append((t2 - t) / 1e3)
        t = t2
    ring = np.zeros((len(recs) + 7, 4), dtype=np.uint64)   # empty slots are dropped
    ring[:len(recs)] = np.array(recs, dtype=np.uint64)
    d = tr.decode(ring)
    assert len(d["t0"]) == len(recs)
    ls = tr.launches(d)
    assert sum(1 for x in ls if x["kind"] == 3) == 4 * 5
    assert all(x["complete"] for x in ls)
    assert all(x["ctas"] == 24 for x in ls if x["kind"] == 3 and x["gy"] == 6)
    rows = {(r["kind"], r["gy"]): r for r in tr.kind_table(ls)}
    assert rows[(1, 1)]["span_mean_us"] == pytest.approx(30.0)
    assert rows[(6, 1)]["first_wait_us"] == pytest.approx(0.5)
    p = tr.layer_periods(ls)
    assert p["layers"] == 4
    assert p["mean_us"] == pytest.approx(np.mean(periods[:4]))
    assert p["regroup_layers"] == 2 and p["plain_layers"] == 2


def test_traced_library_exports_the_abi_and_the_attach_entry():
    path = os.path.join(ROOT, "tertia_b200", "libqsb200_trace.so")
    if not os.path.exists(path):
        from tertia_b200 import build as qb
        qb.build()
    L = C.CDLL(path)
    for name in header_functions() + ["qs_trace_attach"]:
        assert hasattr(L, name), name
    L.qs_trace_attach.argtypes = [C.c_void_p, C.c_void_p, C.c_uint]
    # the argument checks come before any CUDA call
    assert L.qs_trace_attach(C.c_void_p(16), C.c_void_p(32), 3) == 1   # not a power of two
    assert L.qs_trace_attach(C.c_void_p(16), None, 8) == 1              # no counter
