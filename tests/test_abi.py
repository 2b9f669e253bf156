"""The C ABI library: it loads, exports every symbol include/qsb200.h
declares, and the ctypes mirror of qs_config matches the C layout and
defaults (host-only calls, no GPU needed)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    with open(os.path.join(ROOT, "include", "qsb200.h")) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(qs_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from tertia_b200 import build as qb
    qb.build()
    from tertia_b200.abi import load_library
    return load_library()


def test_exports_every_declared_symbol(lib):
    from tertia_b200.abi import EXPORTED_SYMBOLS
    declared = header_functions()
    assert sorted(EXPORTED_SYMBOLS) == declared
    for name in declared:
        assert hasattr(lib, name), name


def test_config_layout_and_defaults(lib):
    from tertia_b200.abi import QsConfig, default_config
    assert C.sizeof(QsConfig) == 240
    assert QsConfig.seed.offset == 232 and QsConfig.synchrotron.offset == 208
    c = QsConfig()
    assert lib.qs_config_default(C.byref(c)) == 0
    assert c.as_dict() == default_config().as_dict()


def test_status_strings(lib):
    for s in range(10):
        assert lib.qs_status_string(s)
    assert lib.qs_status_string(5).decode() == "too large beam current"


def test_invalid_config_is_rejected_without_touching_the_gpu(lib):
    from tertia_b200.abi import default_config, QS_ERR_INVALID
    h = C.c_void_p()
    bad = default_config(ny=12)
    assert lib.qs_create(C.byref(bad), C.byref(h)) == QS_ERR_INVALID
    assert b"multiples of 8" in lib.qs_last_error(None)


class _FakePackLib:
    """Stands in for the two hand-off calls of the library (host only)."""

    def __init__(self, n):
        self.n = n
        self.calls = []

    def qs_layer_pack_size(self, h):
        return self.n

    def qs_pack_layer(self, h, ptr, n):
        self.calls.append(n)
        a = C.cast(ptr, C.POINTER(C.c_double))
        for i in range(n):
            a[i] = float(i)
        return 0


def _fake_mesh(n):
    from tertia_b200.mesh import Mesh
    m = Mesh.__new__(Mesh)
    m._L = _FakePackLib(n)
    m._h = C.c_void_p(1)
    return m


def test_pack_layer_fills_a_given_buffer_in_place():
    import numpy as np
    m = _fake_mesh(24)
    assert m.pack_size() == 24
    out = np.zeros(24)
    got = m.pack_layer(out=out)
    assert got is out and np.array_equal(out, np.arange(24.0))
    assert np.array_equal(m.pack_layer(), np.arange(24.0))
    for bad in (np.zeros(23), np.zeros(24, dtype=np.float32), np.zeros(48)[::2]):
        with pytest.raises(ValueError):
            m.pack_layer(out=bad)
    assert m._L.calls == [24, 24]
    m._h = None   # nothing to destroy
