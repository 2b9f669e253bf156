"""Layer output (qs_save_fields / qs_save_movie_frame, the reference's
Mesh::Save field file and movie frames, save.cpp:520-838, mesh.cpp:976-1090)
in the QSF1 layout: the reader on a file built to the layout by hand (host),
and on the GPU the files against the field store read plane by plane."""
import numpy as np
import pytest

from tertia_b200 import workload as wl
from tertia_b200.fields_io import read_qsf, write_qsf


def test_reader_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    data = {"meshinfo": np.arange(16, dtype=np.int32), "phase": np.array([0.5]),
            "X": np.linspace(0, 1, 7), "Ex": rng.standard_normal((3, 5, 7))}
    p = tmp_path / "f.qsf"
    write_qsf(p, data)
    got = read_qsf(p)
    assert set(got) == set(data)
    for k, v in data.items():
        assert got[k].dtype == v.dtype and np.array_equal(got[k], v), k
    raw = p.read_bytes()
    assert raw[:8] == b"QSF1\0\0\0\0"
    # the layer index fastest: Ex[k, j, i] is stored at i + 7 (j + 5 k)
    off = int(np.frombuffer(raw, "<i8", 1, 16 + 3 * 72 + 64)[0])
    flat = np.frombuffer(raw, "<f8", 105, off)
    assert flat[2 + 7 * (1 + 5 * 2)] == data["Ex"][2, 1, 2]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_saved_fields_are_the_field_store(tmp_path, prec):
    from tertia_b200.abi import PRECISIONS
    from tertia_b200.mesh import Mesh
    cfg = wl.small_config(n=32, layers=24)
    cfg.ny = 64                     # ny != nz, so the axes cannot be confused
    cfg.precision = PRECISIONS[prec]
    cfg.store_sources = 1
    with Mesh(cfg) as m:
        m.load_beam(wl.small_beam(cfg, n=3000))
        m.load_front_plasma(wl.front_plasma(cfg, seed=2))
        m.step()
        m.save_fields(tmp_path / "f.qsf")
        m.save_movie_frame(tmp_path / "m.qsf")
        planes = {f: np.stack([m.get_field3d(f, i) for i in range(cfg.nx)])
                  for f in range(10)}        # [i, k, j]
        phase = m.get_phase()
    f = read_qsf(tmp_path / "f.qsf")
    names = ["Ex", "Ey", "Ez", "Bx", "By", "Bz", "Jx", "Jy", "Jz", "Dens"]
    assert list(f["meshinfo"][:12]) == [cfg.nx, 0, cfg.nx, 0, cfg.ny, 0, cfg.ny, 0, cfg.nz, 0,
                                        cfg.nz, 0]
    assert f["phase"][0] == phase
    np.testing.assert_allclose(f["X"], np.arange(cfg.nx) * cfg.hx + phase)
    np.testing.assert_allclose(f["Y"], np.arange(cfg.ny) * cfg.hy - cfg.ny * cfg.hy / 2)
    np.testing.assert_allclose(f["Z"], np.arange(cfg.nz) * cfg.hz - cfg.nz * cfg.hz / 2)
    for q, name in enumerate(names):
        want = np.transpose(planes[q], (1, 2, 0))              # [k, j, i]
        assert f[name].shape == (cfg.nz, cfg.ny, cfg.nx)
        assert np.array_equal(f[name], want), name
    assert np.max(np.abs(f["Ex"])) > 1e-3
    mv = read_qsf(tmp_path / "m.qsf")
    for q, name in enumerate(names):
        assert np.array_equal(mv[name + "_xy"], planes[q][:, cfg.nz // 2, :].T), name
        assert np.array_equal(mv[name + "_xz"], planes[q][:, :, cfg.ny // 2].T), name
