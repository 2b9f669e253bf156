"""Shared helpers of the GPU parity tests."""
import numpy as np

from tertia_b200 import workload as wl
from tertia_b200.abi import PRECISIONS


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return d / n if n > 0 else d


def cfg_for(prec, **kw):
    c = wl.small_config(**kw)
    c.precision = PRECISIONS[prec]
    return c


def run_pair(oracle_lib, cfg, beam, fronts, steps=1):
    """Run `steps` full steps (beam push + march) in the oracle and on the
    GPU from identical inputs; returns (oracle, mesh)."""
    from tertia_b200.mesh import Mesh
    o = oracle_lib.Oracle(cfg)
    m = Mesh(cfg)
    o.load_beam(beam)
    m.load_beam(beam)
    for s in range(steps):
        o.load_front_plasma(fronts[s])
        m.load_front_plasma(fronts[s])
        o.step()
        m.step()
    return o, m
