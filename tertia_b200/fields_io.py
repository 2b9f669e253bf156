"""Reader of the QSF1 layer-output files (qs_save_fields, qs_save_movie_frame).

QSF1 carries the datasets of the reference's HDF5 field file (Mesh::Save,
save.cpp:520-838) and of its movie frames (Mesh::SaveCadrMovie2,
mesh.cpp:976-1090) in a plain self-describing layout, little-endian:

    bytes 0-7   b"QSF1" and four zero bytes
    int32 ndatasets, int32 0
    ndatasets entries of 72 bytes: name[32] (zero padded), int32 dtype
    (1 int32, 2 float64), int32 rank, int64 dims[3] (fastest first, unused
    ones 1), int64 byte offset of the data
    the data blocks

read_qsf returns {name: numpy array}; a 3-D field of dims (nx, ny, nz) comes
back as an array indexed [k, j, i] (the layer index i fastest, as stored).
"""
from __future__ import annotations

import numpy as np

MAGIC = b"QSF1\0\0\0\0"
ENTRY = np.dtype([("name", "S32"), ("dtype", "<i4"), ("rank", "<i4"), ("dims", "<i8", (3,)),
                  ("offset", "<i8")])


def read_qsf(path) -> dict:
    with open(path, "rb") as f:
        raw = f.read()
    if raw[:8] != MAGIC:
        raise ValueError(f"{path}: not a QSF1 file")
    n = int(np.frombuffer(raw, "<i4", 1, 8)[0])
    table = np.frombuffer(raw, ENTRY, n, 16)
    out = {}
    for e in table:
        dt = {1: np.dtype("<i4"), 2: np.dtype("<f8")}[int(e["dtype"])]
        dims = [int(d) for d in e["dims"]]
        count = dims[0] * dims[1] * dims[2]
        a = np.frombuffer(raw, dt, count, int(e["offset"])).copy()
        shape = tuple(reversed(dims[: int(e["rank"])]))
        out[e["name"].decode().rstrip("\0")] = a.reshape(shape)
    return out


def write_qsf(path, datasets: dict):
    """Write {name: array} as QSF1 (int32 or float64; an array [k, j, i] is
    stored with i fastest): the layout the library writes, for tests and
    tools."""
    items = []
    for name, a in datasets.items():
        a = np.ascontiguousarray(a)
        dtype = 1 if a.dtype == np.int32 else 2
        a = a.astype("<i4" if dtype == 1 else "<f8")
        dims = list(reversed(a.shape)) + [1] * (3 - a.ndim)
        items.append((name, dtype, a.ndim, dims, a))
    pos = 16 + 72 * len(items)
    table = np.zeros(len(items), ENTRY)
    for t, (name, dtype, rank, dims, a) in enumerate(items):
        table[t] = (name.encode(), dtype, rank, dims, pos)
        pos = (pos + a.nbytes + 7) & ~7
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(np.array([len(items), 0], "<i4").tobytes())
        f.write(table.tobytes())
        for t, (_, _, _, _, a) in enumerate(items):
            f.seek(int(table[t]["offset"]))
            f.write(a.tobytes())
