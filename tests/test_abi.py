"""The C ABI library: it loads, exports every symbol include/qsb200.h
declares, and the ctypes mirror of qs_config matches the C layout and
defaults (host-only calls, no GPU needed)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "qsb200.h")).read()
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
