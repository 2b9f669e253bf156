"""The traced library (libqsb200_trace.so) on the GPU: a short march with the
ring attached records every instrumented kernel kind with ordered stamps, and
marches like libqsb200.so.  Each library runs in a process of its own."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PLAIN = r"""
import sys
import numpy as np
sys.path.insert(0, {root!r})
from tertia_b200 import workload as wl
from tertia_b200.abi import QS_SHAPE_CIC
from tertia_b200.mesh import Mesh
w = wl.make_workload("c1", "fp32")
cfg = w.cfg
cfg.shape = QS_SHAPE_CIC
cfg.ny = cfg.nz = 128
cfg.nx = 48
beam = wl.sample_beam(cfg, wl.BeamSpec(100_000, nb_over_n0=1e-4))
with Mesh(cfg) as m:
    m.load_beam(beam)
    for _ in range(3):
        m.step()
    np.save({out!r}, m.onaxis_ex())
"""


@pytest.mark.gpu
def test_traced_march_records_and_matches_the_plain_library(tmp_path):
    pre = str(tmp_path / "t")
    # one warm-up, one untraced and one traced step: three steps, as PLAIN
    r = subprocess.run([sys.executable, "-m", "tertia_b200.trace", "--grid", "128", "--layers",
                        "48", "--warmup", "1", "--records", "65536", "--keep", "65536",
                        "--out", pre, "--onaxis", pre + "_ex.npy"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "layer period" in r.stdout
    from tertia_b200 import trace as tr
    d = tr.decode(np.load(pre + "_rec.npy"))
    assert len(d["t0"]) > 0
    assert np.all(d["t0"] <= d["t1"]) and np.all(d["t1"] <= d["t2"])
    kinds = set(d["kind"].tolist())
    assert {1, 2, 3, 6, 8, 10, 11} <= kinds, kinds
    p = tr.layer_periods(tr.launches(d))
    assert p["layers"] >= 40 and p["mean_us"] > 0
    out = str(tmp_path / "plain_ex.npy")
    r = subprocess.run([sys.executable, "-c", PLAIN.format(root=ROOT, out=out)], cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    a, b = np.load(pre + "_ex.npy"), np.load(out)
    # FP32 atomic deposits differ in their last bits from run to run
    assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b)
