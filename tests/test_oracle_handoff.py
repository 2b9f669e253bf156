"""The xi-pipeline hand-off in the oracle (PackLayer / UnpackLayer,
para.cpp:94-285): the buffer layout, and a march split over two boxes, the
second starting from the layer the first one packed, against one march over
the whole box.  Host only."""
import numpy as np
import pytest

from tertia_b200 import workload as wl
from tertia_b200.abi import QS_F_EX, QS_F_BZ, QS_F_JX


def box_pair(L=12, n=16):
    full = wl.small_config(n=n, layers=2 * L, ts=0.0, synchrotron=0, pspread_x=0.01,
                           pspread_y=0.01, pspread_z=0.01)
    half = wl.small_config(n=n, layers=L, ts=0.0, synchrotron=0, pspread_x=0.01,
                           pspread_y=0.01, pspread_z=0.01)
    beam = wl.small_beam(full, n=3000)
    # the driver stays in the upper box: its deposit (layers i, i+1) never
    # reaches the lower box, and layer L carries beam current for the hand-off
    keep = beam["i"] >= L
    beam = {k: v[keep] for k, v in beam.items()}
    upper = dict(beam)
    upper["i"] = (beam["i"] - L).astype(np.int32)
    empty = {k: v[:0] for k, v in beam.items()}
    return full, half, beam, upper, empty


def split_layout(buf, cfg):
    P = cfg.ny * cfg.nz
    m = (buf.size - 12 * P) // 12
    planes = buf[:12 * P].reshape(12, P)
    parts = buf[12 * P:].reshape(12, m)
    return planes, parts


def sorted_particles(parts):
    # the order within a cell is the list order; compare as sets per cell
    key = np.lexsort((parts[3], parts[4], parts[5], parts[0], parts[9] + 1e6 * parts[10]))
    return parts[:, key]


def test_pack_layout(oracle_lib):
    full, half, beam, upper, empty = box_pair()
    o = oracle_lib.Oracle(half)
    o.load_beam(upper)
    o.load_front_plasma(wl.front_plasma(half, seed=3))
    o.step()
    buf = o.pack_layer()
    planes, parts = split_layout(buf, half)
    P = half.ny * half.nz
    assert buf.size == 12 * P + 12 * P * half.ppc
    # Bx By Bz Ex Ey Ez Jx Jy Jz Rho
    for slot, f in zip(range(6), (3, 4, 5, 0, 1, 2)):
        np.testing.assert_array_equal(planes[slot], o.get_field3d(f, 0).ravel())
    assert np.max(np.abs(planes[3])) > 0 and np.max(np.abs(planes[10])) > 0
    pl = o.get_plasma()
    cells = (parts[9] + half.ny * parts[10]).astype(np.int64)
    assert np.all(np.diff(cells) >= 0)                        # cell by cell
    np.testing.assert_array_equal(np.sort(cells), np.sort(pl["cell"]))
    np.testing.assert_array_equal(np.sort(parts[7]), np.sort(pl["w"]))
    assert np.all(parts[6] == half.plasma_q2m) and np.all(parts[11] == 0) and np.all(parts[8] == 0)
    o.close()


def test_two_boxes_equal_one_box(oracle_lib):
    full, half, beam, upper, empty = box_pair()
    front = wl.front_plasma(half, seed=3)
    whole = oracle_lib.Oracle(full)
    whole.load_beam(beam)
    whole.load_front_plasma(front)
    whole.step()
    up = oracle_lib.Oracle(half)
    up.load_beam(upper)
    up.load_front_plasma(front)
    up.step()
    lo = oracle_lib.Oracle(half)
    lo.load_beam(empty)
    lo.unpack_layer(up.pack_layer())
    lo.step()
    L = half.nx
    ex = whole.onaxis_ex()
    assert np.max(np.abs(ex[:L])) > 1e-3                      # the wake reached the lower box
    np.testing.assert_allclose(lo.onaxis_ex(), ex[:L], rtol=0, atol=1e-13 * np.max(np.abs(ex)))
    np.testing.assert_allclose(up.onaxis_ex(), ex[L:], rtol=0, atol=1e-13 * np.max(np.abs(ex)))
    for f in (QS_F_EX, QS_F_BZ, QS_F_JX):
        for i in (0, L // 2, L - 1):
            a, b = lo.get_field3d(f, i).ravel(), whole.get_field3d(f, i).ravel()
            assert np.max(np.abs(a - b)) <= 1e-12 * max(np.max(np.abs(b)), 1e-30), (f, i)
    # the plasma leaving the lower box is the plasma leaving the whole box
    pa = sorted_particles(split_layout(lo.pack_layer(), half)[1])
    pb = sorted_particles(split_layout(whole.pack_layer(), full)[1])
    np.testing.assert_allclose(pa, pb, rtol=1e-12, atol=1e-14)
    for o in (whole, up, lo):
        o.close()


def test_without_a_received_layer_the_box_starts_empty(oracle_lib):
    """The received layer serves one march; the next starts from the empty
    front, like a box that never received one."""
    full, half, beam, upper, empty = box_pair()
    front = wl.front_plasma(half, seed=3)
    up = oracle_lib.Oracle(half)
    up.load_beam(upper)
    up.load_front_plasma(front)
    up.step()
    lo = oracle_lib.Oracle(half)
    lo.load_beam(upper)
    lo.unpack_layer(up.pack_layer())
    lo.step()
    assert np.max(np.abs(lo.onaxis_ex() - up.onaxis_ex())) > 1e-6
    # march again over the beam currents of the first step (no beam push)
    for o in (up, lo):
        o.load_front_plasma(front)
        o.move_all_split_layers()
    np.testing.assert_array_equal(lo.onaxis_ex(), up.onaxis_ex())
    for o in (up, lo):
        o.close()
