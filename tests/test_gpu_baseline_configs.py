"""Parity on the benchmark's own configurations, against the oracle.

c0, exactly as the benchmark states it: 128 x 128 transverse cells of 0.05,
256 layers of 0.05, uniform plasma with 4 particles per cell on the
reference lattice and zero momentum, a bi-Gaussian electron driver
(sigma_r 0.5, sigma_xi 1.0, peak n_b/n_0 0.5, gamma 1000) of 1e5 particles
sampled from a seed, CIC deposit, one beam step.  A second beam step then
pushes the beam through the first march's fields, for its phase space.

c1 head segment: the 512 x 512 grid of c1 (cells of 0.05, 4 ppc, thermal
spread 0.01) over the 64 layers behind the front, with the part of c1's
1e6-particle driver that lies in those layers, two beam steps.

Each is run once in the oracle (FP64) and compared with the GPU path in FP64
(dense-matrix transforms and FFT transforms) and in FP32.  Asserted: on-axis Ez (the reference's longitudinal Ex) and the
full layers of all six fields, psi, the beam phase space (cells, in-cell
fractions and momenta), the plasma cells after the march (bit-exact in
FP64), and the FP64 charge sums of every layer.
"""
import os

import numpy as np
import pytest

from tertia_b200 import workload as wl
from tertia_b200.abi import PRECISIONS, QS_SHAPE_CIC
from gpu_helpers import rel_l2

pytestmark = pytest.mark.gpu

# relative L2 tolerances against the FP64 oracle: FP64 agrees to rounding;
# the FP32 path is held to the 1e-5 that the benchmark sets for Ez
TOL = {"fp64": 1e-10, "fp64fft": 1e-10, "fp32": 1e-5}


def c0_case():
    w = wl.make_workload("c0")
    cfg = w.cfg
    beam = wl.workload_beam(w)
    fronts = [wl.front_plasma(cfg, seed=s, thermal=False) for s in (1, 2)]
    return cfg, beam, fronts


def c1_head_case(layers=64):
    """c1's grid and driver over the `layers` layers behind the front."""
    w = wl.make_workload("c1")
    full = w.cfg
    beam = wl.workload_beam(w)
    keep = beam["i"] >= full.nx - layers
    beam = {k: np.ascontiguousarray(v[keep]) for k, v in beam.items()}
    beam["i"] = (beam["i"] - (full.nx - layers)).astype(np.int32)
    cfg = full.copy()
    cfg.nx = layers
    cfg.shape = QS_SHAPE_CIC
    fronts = [wl.front_plasma(cfg, seed=s) for s in (3, 4)]
    return cfg, beam, fronts


def summary(obj, cfg, first):
    """What the comparison reads after a beam step (the full layers and the
    plasma after the first step only)."""
    out = {"ex": obj.onaxis_ex(), "psi": obj.psi(), "beam": obj.get_beam(),
           "sums": obj.charge_sums()}
    if first:
        out["fields"] = np.stack([np.stack([obj.get_field3d(f, i) for f in range(6)])
                                  for i in range(cfg.nx)])
        out["plasma"] = obj.get_plasma()
    return out


def run_two_steps(make, cfg, beam, fronts):
    m = make(cfg)
    m.load_beam(beam)
    out = []
    for s, f in enumerate(fronts):
        m.load_front_plasma(f)
        m.step()
        out.append(summary(m, cfg, s == 0))
    m.close()
    return out


@pytest.fixture(scope="module", params=["c0", "c1_head"])
def case(request, oracle_lib):
    oracle_lib.set_threads(os.cpu_count() or 1)
    cfg, beam, fronts = c0_case() if request.param == "c0" else c1_head_case()
    ref = run_two_steps(oracle_lib.Oracle, cfg, beam, fronts)
    return request.param, cfg, beam, fronts, ref


def check_step(prec, cfg, got, ref, first):
    tol = TOL[prec]
    assert np.max(np.abs(ref["ex"])) > 1e-2          # a wake was driven
    errs = {
        "ez_onaxis": rel_l2(got["ex"], ref["ex"]),
        "psi": rel_l2(got["psi"], ref["psi"]),
        "ez_full_layers": rel_l2(got["fields"][:, 0], ref["fields"][:, 0]),
        "fields": rel_l2(got["fields"], ref["fields"]),
    }
    for q in ("rho", "jx", "rho_beam"):
        a, b = got["sums"][q], ref["sums"][q]
        errs["sum_" + q] = float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
    print(prec, "step 1" if first else "step 2", {k: f"{v:.2e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < tol, (k, v)
    po, pm = ref["plasma"], got["plasma"]
    if prec.startswith("fp64"):
        assert np.array_equal(pm["cell"], po["cell"])
    else:
        assert np.mean(pm["cell"] == po["cell"]) > 0.999
    assert np.any(po["cell"] != np.repeat(np.arange(cfg.ny * cfg.nz), cfg.ppc))   # moved
    for k in ("px", "py", "pz"):
        assert rel_l2(pm[k], po[k]) < tol * 10, k


def check_beam(prec, beam, got, ref):
    bo, bm = ref["beam"], got["beam"]
    for k in ("i", "j", "k"):
        if prec.startswith("fp64"):
            assert np.array_equal(bm[k], bo[k]), k
        else:
            assert np.mean(bm[k] == bo[k]) > 0.9999, k
    # the kicks of the two pushes: momentum changes, relative L2
    for k in ("px", "py", "pz"):
        d_o = np.asarray(bo[k]) - np.asarray(beam[k])
        d_m = np.asarray(bm[k]) - np.asarray(beam[k])
        assert np.linalg.norm(d_o) > 0, k
        assert rel_l2(d_m, d_o) < TOL[prec] * (1 if prec.startswith("fp64") else 10), k
    same = np.asarray(bm["i"]) == np.asarray(bo["i"])
    for k in ("x", "y", "z"):
        np.testing.assert_allclose(np.asarray(bm[k])[same], np.asarray(bo[k])[same],
                                   rtol=0, atol=1e-12 if prec.startswith("fp64") else 1e-6)


@pytest.mark.parametrize("prec", ["fp64", "fp64fft", "fp32"])
def test_baseline_config_matches_oracle(case, prec):
    from tertia_b200.mesh import Mesh
    name, cfg0, beam, fronts, ref = case
    cfg = cfg0.copy()
    cfg.precision = PRECISIONS[prec]
    got = run_two_steps(Mesh, cfg, beam, fronts)
    check_step(prec, cfg, got[0], ref[0], True)
    check_beam(prec, beam, got[1], ref[1])
    # after the second step the fields follow from the moved beam as well
    assert rel_l2(got[1]["ex"], ref[1]["ex"]) < TOL[prec]
