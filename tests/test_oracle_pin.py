"""The oracle's push and beam push against the reference's own code.

oracle/_ref/librefpin.so is the reference's Mesh::MoveParticlesLayerSplit
(movepart_splitlayer.cpp:781-1544) with ExchangeCurrentsSplit (:1685-1711)
and its Mesh::MoveBeamParticles with MoveBeamInCell (movebeam.cpp:14-774),
compiled from the reference checkout by oracle/Makefile (target refpin) and
driven by oracle/ref_pin.cpp.  On identical decks and particles the oracle's
restatements (qso_push_layer_f64, the oracle's beam push) must give the same
particle states and cells bit for bit, and the same deposits up to the order
of the additions (the reference adds the guard ring after the push, the
oracle folds each deposit as it is made).

Host only; skipped where the pin library was not built (no reference
checkout to compile it from).
"""
import os

import numpy as np
import pytest

from tertia_b200 import workload as wl
from tertia_b200.abi import QS_F_JXBEAM, QS_F_RHOBEAM


@pytest.fixture(scope="module")
def ref(oracle_lib):
    oracle_lib.build_reference()
    L = oracle_lib.refpin_lib()
    if L is None:
        pytest.skip("the reference's push was not built here (no reference checkout)")
    return L


def plasma_deck(n=16, hx=0.05, hy=0.05, spread=0.05, bext=(0.0, 0.0, 0.0), seed=3):
    cfg = wl.small_config(n=n, layers=4, h=hy, hx=hx, pspread_x=spread, pspread_y=spread,
                          pspread_z=spread)
    cfg.bx_ext, cfg.by_ext, cfg.bz_ext = bext
    rng = np.random.default_rng(seed)
    front = wl.front_plasma(cfg, seed=seed)
    # off-lattice in-cell positions, so that particles cross cell edges
    front["y"] = rng.uniform(0.0, 1.0, len(front["y"]))
    front["z"] = rng.uniform(0.0, 1.0, len(front["z"]))
    plane = cfg.ny * cfg.nz
    P = 0.2 * rng.standard_normal((6, plane))
    C = P + 0.02 * rng.standard_normal((6, plane))
    return cfg, front, P, C


def run_reference_push(L, cfg, f, P, C, full):
    n = len(f["y"])
    cell = np.ascontiguousarray(f["cell"], dtype=np.int32)
    arr = {k: np.ascontiguousarray(f[k], dtype=np.float64).copy()
           for k in ("y", "z", "px", "py", "pz", "w")}
    dep = np.zeros(4 * cfg.ny * cfg.nz)
    cell_out = np.full(n, -1, dtype=np.int32)
    st = L.refpin_push_layer(cfg, n, cell, arr["y"], arr["z"], arr["px"], arr["py"], arr["pz"],
                             arr["w"], np.ascontiguousarray(P.reshape(-1)),
                             np.ascontiguousarray(C.reshape(-1)), dep, cell_out, int(full))
    assert st == 0
    return arr, dep.reshape(4, cfg.nz, cfg.ny), cell_out


@pytest.mark.parametrize("full", [0, 1])
@pytest.mark.parametrize("case", ["thermal", "subcycled", "external_b"])
def test_plasma_push_matches_reference(oracle_lib, ref, case, full):
    if case == "thermal":
        deck = plasma_deck()
    elif case == "subcycled":      # |dy| above a cell per layer: the sub-stepped move
        deck = plasma_deck(hx=0.2, hy=0.02, spread=0.4)
    else:
        deck = plasma_deck(spread=0.1, bext=(0.3, -0.2, 0.1))
    cfg, f, P, C = deck
    got, dep, cell_out = run_reference_push(ref, cfg, f, P, C, full)
    o = oracle_lib.push_layer(cfg, f["cell"], f["y"], f["z"], f["px"], f["py"], f["pz"], f["w"],
                              P, C, full=bool(full), precise=False)
    scale = np.max(np.abs(dep))
    assert scale > 0
    np.testing.assert_allclose(o["dep"], dep, rtol=0, atol=1e-13 * scale)
    if full:
        for k in ("y", "z", "px", "py", "pz"):
            assert np.array_equal(o[k], got[k]), k          # bit for bit
        # the live NGP path relinks a particle into its own cell (the outer j,
        # k at :1501-1512), whatever cell its sub-steps deposited into
        assert np.array_equal(o["cell"], cell_out)
        assert np.array_equal(cell_out, f["cell"])
    if case == "subcycled":
        assert np.mean(o["dep_cell"] != f["cell"]) > 0.2     # the deposits moved on


def beam_deck(n=16, layers=12, synchrotron=1, seed=5):
    cfg = wl.small_config(n=n, layers=layers, h=0.2, hx=0.1)
    cfg.synchrotron = synchrotron
    cfg.beam_polarity = 1.0          # the reference takes the species' polarity, 1 for electrons
    cfg.ts = 2.0
    rng = np.random.default_rng(seed)
    nb = 3000
    beam = {"i": rng.integers(0, layers, nb).astype(np.int32),
            "j": rng.integers(0, n, nb).astype(np.int32),
            "k": rng.integers(0, n, nb).astype(np.int32),
            "x": rng.uniform(0, 1, nb), "y": rng.uniform(0, 1, nb), "z": rng.uniform(0, 1, nb),
            "px": 1000.0 + 10.0 * rng.standard_normal(nb),
            "py": 0.5 * rng.standard_normal(nb), "pz": 0.5 * rng.standard_normal(nb),
            "w": rng.uniform(0.5, 1.5, nb)}
    # group by cell in the reference's list order is not needed: every
    # particle is pushed independently; sort by (i, j, k) for the lists
    fields = 0.3 * rng.standard_normal((layers + 1, 6, n * n))
    return cfg, beam, fields


@pytest.mark.parametrize("synchrotron", [0, 1])
def test_beam_push_matches_reference(oracle_lib, ref, synchrotron, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)        # the reference writes hostBeamFile.dat here
    cfg, beam, fields = beam_deck(synchrotron=synchrotron)
    nb = len(beam["x"])
    b = {k: np.ascontiguousarray(v).copy() for k, v in beam.items()}
    cur = np.zeros((cfg.nx + 1) * 4 * cfg.ny * cfg.nz)
    st = ref.refpin_beam_push(cfg, nb, b["i"], b["j"], b["k"], b["x"], b["y"], b["z"], b["px"],
                              b["py"], b["pz"], b["w"], np.ascontiguousarray(fields.reshape(-1)),
                              cur)
    assert st == 0
    cur = cur.reshape(cfg.nx + 1, 4, cfg.nz, cfg.ny)
    o = oracle_lib.Oracle(cfg)
    for i in range(cfg.nx + 1):
        for fld in range(6):
            o.set_field3d(fld, i, fields[i, fld])
    o.load_beam(beam)
    o.move_beam_particles()
    ob = o.get_beam()
    for k in ("i", "j", "k", "x", "y", "z", "px", "py", "pz"):
        assert np.array_equal(np.asarray(ob[k]), b[k]), k        # bit for bit
    assert np.max(np.abs(ob["py"] - beam["py"])) > 1e-3          # the fields kicked the beam
    if synchrotron:
        # the radiation loss is on: the reference's and the oracle's agree
        assert np.all(ob["px"] != beam["px"])
    for fld, q in ((QS_F_RHOBEAM, 3), (QS_F_JXBEAM, 0)):
        got = np.stack([o.get_beam_currents(fld, i) for i in range(cfg.nx + 1)])
        want = cur[:, q]
        scale = np.max(np.abs(want))
        assert scale > 0
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-13 * scale)
