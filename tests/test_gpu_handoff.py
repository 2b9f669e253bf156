"""The xi-pipeline hand-off on the GPU (qs_pack_layer / qs_unpack_layer, the
reference's PackLayer / UnpackLayer, para.cpp:94-285) against the oracle: the
packed tail layer, a march that starts from a received layer, and a march
split over two boxes against one march over the whole box."""
import numpy as np
import pytest

from tertia_b200 import abi
from tertia_b200 import workload as wl
from gpu_helpers import cfg_for, rel_l2

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp64fft": 1e-10, "fp32": 5e-4}


def boxes(prec, shape, L=12, n=32):
    kw = dict(n=n, ts=0.0, synchrotron=0, pspread_x=0.01, pspread_y=0.01, pspread_z=0.01,
              shape=shape)
    full = cfg_for(prec, layers=2 * L, **kw)
    half = cfg_for(prec, layers=L, **kw)
    beam = wl.small_beam(full, n=4000)
    keep = beam["i"] >= L          # the driver stays in the upper box
    beam = {k: v[keep] for k, v in beam.items()}
    upper = dict(beam)
    upper["i"] = (beam["i"] - L).astype(np.int32)
    empty = {k: v[:0] for k, v in beam.items()}
    return full, half, beam, upper, empty


def layout(buf, cfg):
    P = cfg.ny * cfg.nz
    m = (buf.size - 12 * P) // 12
    return buf[:12 * P].reshape(12, P), buf[12 * P:].reshape(12, m)


def by_cell(parts):
    key = np.lexsort((parts[5], parts[4], parts[0], parts[9] + 1e6 * parts[10]))
    return parts[:, key]


@pytest.mark.parametrize("prec,shape", [("fp64", abi.QS_SHAPE_NGP), ("fp64", abi.QS_SHAPE_CIC),
                                        ("fp64fft", abi.QS_SHAPE_CIC), ("fp32", abi.QS_SHAPE_CIC)])
def test_packed_layer_matches_oracle(oracle_lib, prec, shape):
    from tertia_b200.mesh import Mesh
    full, half, beam, upper, empty = boxes(prec, shape)
    front = wl.front_plasma(half, seed=5)
    o, m = oracle_lib.Oracle(half), Mesh(half)
    for h in (o, m):
        h.load_beam(upper)
        h.load_front_plasma(front)
        h.step()
    bo, bm = o.pack_layer(), m.pack_layer()
    assert bm.size == bo.size
    po, qo = layout(bo, half)
    pm, qm = layout(bm, half)
    for slot in range(12):
        assert np.max(np.abs(po[slot])) > 0, slot
        assert rel_l2(pm[slot], po[slot]) < TOL[prec] * (10 if slot >= 6 else 1), slot
    cm = qm[9] + half.ny * qm[10]
    assert np.all(np.diff(cm) >= 0)                            # cell by cell
    if prec in ("fp64", "fp64fft"):
        np.testing.assert_allclose(by_cell(qm), by_cell(qo), rtol=1e-9, atol=1e-11)
    else:
        np.testing.assert_array_equal(np.sort(qm[7]), np.sort(qo[7]).astype(np.float32))
        assert np.mean(np.sort(cm) == np.sort(qo[9] + half.ny * qo[10])) > 0.99
    o.close()
    m.close()


@pytest.mark.parametrize("prec,shape", [("fp64", abi.QS_SHAPE_NGP), ("fp64", abi.QS_SHAPE_CIC),
                                        ("fp64fft", abi.QS_SHAPE_CIC), ("fp32", abi.QS_SHAPE_CIC)])
def test_packed_particles_are_the_plasma_cell_by_cell(prec, shape):
    """The particle blocks hold the plasma in flight ordered by cell (k outer,
    j inner) and by load order within a cell, value for value, and the planes
    are the tail layer's fields."""
    from tertia_b200.mesh import Mesh
    full, half, beam, upper, empty = boxes(prec, shape)
    with Mesh(half) as m:
        m.load_beam(upper)
        m.load_front_plasma(wl.front_plasma(half, seed=5))
        m.step()
        buf = m.pack_layer()
        pl = m.get_plasma()
        planes, parts = layout(buf, half)
        for slot, f in zip(range(6), (abi.QS_F_BX, abi.QS_F_BY, abi.QS_F_BZ, abi.QS_F_EX,
                                      abi.QS_F_EY, abi.QS_F_EZ)):
            np.testing.assert_array_equal(planes[slot], m.get_field3d(f, 0).ravel())
    order = np.argsort(pl["cell"], kind="stable")
    n = order.size
    assert parts.shape == (12, n)
    for row, key in ((0, "px"), (1, "py"), (2, "pz"), (4, "y"), (5, "z"), (7, "w")):
        np.testing.assert_array_equal(parts[row], pl[key][order], err_msg=key)
    cell = pl["cell"][order]
    np.testing.assert_array_equal(parts[9], cell % half.ny)
    np.testing.assert_array_equal(parts[10], cell // half.ny)
    assert np.all(parts[3] == 0) and np.all(parts[8] == 0) and np.all(parts[11] == 0)
    assert np.all(parts[6] == half.plasma_q2m)


@pytest.mark.parametrize("prec,shape,graph", [("fp64", abi.QS_SHAPE_NGP, 1),
                                              ("fp64", abi.QS_SHAPE_CIC, 0),
                                              ("fp64fft", abi.QS_SHAPE_CIC, 1),
                                              ("fp32", abi.QS_SHAPE_CIC, 1)])
def test_march_from_a_received_layer_matches_oracle(oracle_lib, prec, shape, graph):
    from tertia_b200.mesh import Mesh
    full, half, beam, upper, empty = boxes(prec, shape)
    half.use_graph = graph
    up = oracle_lib.Oracle(half)
    up.load_beam(upper)
    up.load_front_plasma(wl.front_plasma(half, seed=5))
    up.step()
    buf = up.pack_layer()
    o, m = oracle_lib.Oracle(half), Mesh(half)
    for h in (o, m):
        h.load_beam(empty)
        h.unpack_layer(buf)
        h.step()
    e_o, e_m = o.onaxis_ex(), m.onaxis_ex()
    assert np.max(np.abs(e_o)) > 1e-3
    assert rel_l2(e_m, e_o) < TOL[prec]
    for f in (abi.QS_F_EX, abi.QS_F_EY, abi.QS_F_BZ):
        a = np.stack([m.get_field3d(f, i) for i in range(half.nx)])
        b = np.stack([o.get_field3d(f, i) for i in range(half.nx)])
        assert rel_l2(a, b) < TOL[prec] * 10, f
    for h in (up, o, m):
        h.close()


def test_two_boxes_equal_one_box():
    from tertia_b200.mesh import Mesh
    full, half, beam, upper, empty = boxes("fp64", abi.QS_SHAPE_NGP)
    front = wl.front_plasma(half, seed=5)
    whole, up, lo = Mesh(full), Mesh(half), Mesh(half)
    whole.load_beam(beam)
    whole.load_front_plasma(front)
    whole.step()
    up.load_beam(upper)
    up.load_front_plasma(front)
    up.step()
    lo.load_beam(empty)
    lo.unpack_layer(up.pack_layer())
    lo.step()
    L = half.nx
    ex = whole.onaxis_ex()
    assert np.max(np.abs(ex[:L])) > 1e-3
    assert rel_l2(lo.onaxis_ex(), ex[:L]) < 1e-11
    assert rel_l2(up.onaxis_ex(), ex[L:]) < 1e-11
    for h in (whole, up, lo):
        h.close()


def test_received_layer_serves_one_march():
    """The received layer is the front of the next march only; the captured
    march is rebuilt when the front changes between received and empty."""
    from tertia_b200.mesh import Mesh
    full, half, beam, upper, empty = boxes("fp64", abi.QS_SHAPE_NGP)
    front = wl.front_plasma(half, seed=5)
    up, lo = Mesh(half), Mesh(half)
    for h in (up, lo):
        h.load_beam(upper)
        h.load_front_plasma(front)
    up.step()
    buf = up.pack_layer()
    lo.unpack_layer(buf)
    lo.step()                         # beam deposit as in up's step, received front
    e1 = lo.onaxis_ex()
    assert rel_l2(e1, up.onaxis_ex()) > 1e-6
    for h in (up, lo):                # over the same beam currents, empty front
        h.load_front_plasma(front)
        h.move_all_split_layers()
    assert rel_l2(lo.onaxis_ex(), up.onaxis_ex()) < 1e-13
    lo.unpack_layer(buf)              # received again: the first result again
    lo.move_all_split_layers()
    assert rel_l2(lo.onaxis_ex(), e1) < 1e-13
    up.close()
    lo.close()


def test_bad_buffers_are_rejected():
    from tertia_b200.mesh import Mesh
    full, half, beam, upper, empty = boxes("fp64", abi.QS_SHAPE_NGP)
    with Mesh(half) as m:
        with pytest.raises(abi.QsError):
            m.pack_layer()                                     # no march yet
        m.load_beam(upper)
        m.load_front_plasma(wl.front_plasma(half, seed=5))
        m.step()
        buf = m.pack_layer()
        with pytest.raises(abi.QsError):
            m.unpack_layer(buf[:-1])                           # not 12 P + 12 Np
        planes, parts = layout(buf.copy(), half)
        cases = [((9, 0), half.ny, abi.QS_ERR_INVALID, "outside the layer"),        # cell j
                 ((10, 5), 1.5, abi.QS_ERR_INVALID, "outside the layer"),           # k not whole
                 ((4, 2), 1.25, abi.QS_ERR_PARTICLE_RANGE, "position"),              # in-cell y
                 ((6, 3), 1.0, abi.QS_ERR_UNSUPPORTED, "species")]                   # Q2m
        for (row, col), value, status, text in cases:
            bad = buf.copy()
            layout(bad, half)[1][row, col] = value
            with pytest.raises(abi.QsError, match=text) as e:
                m.unpack_layer(bad)
            assert e.value.status == status
            assert f"particle {col} " in str(e.value)   # the lowest bad row is named
        # two bad rows: the lower one is reported
        bad = buf.copy()
        layout(bad, half)[1][4, 7] = -0.5
        layout(bad, half)[1][9, 9] = -1.0
        with pytest.raises(abi.QsError, match="particle 7 ") as e:
            m.unpack_layer(bad)
        assert e.value.status == abi.QS_ERR_PARTICLE_RANGE
        m.unpack_layer(buf)
        m.clear_front_layer()
        m.load_front_plasma(wl.front_plasma(half, seed=5))
        m.step()
