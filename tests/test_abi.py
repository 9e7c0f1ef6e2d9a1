"""The C-ABI library loads and exports every symbol include/szp_b200.h
declares (no GPU needed: nothing is called)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "szp_b200.h")).read()
    return sorted(set(re.findall(r"SZP_B200_API\s+[A-Za-z_][A-Za-z_0-9 \*]*?\b([a-z_][a-z_0-9]*)\s*\(", src)))


@pytest.fixture(scope="module")
def libpath():
    import toposzp_b200
    if not os.path.exists(toposzp_b200.LIB_PATH):
        toposzp_b200.build()
    return toposzp_b200.LIB_PATH


def test_library_exports_every_declared_symbol(libpath):
    lib = ctypes.CDLL(libpath)
    syms = declared_symbols()
    assert len(syms) >= 19
    for s in syms:
        assert hasattr(lib, s), s


def test_reference_symbols_present(libpath):
    import toposzp_b200
    lib = ctypes.CDLL(libpath)
    for s in toposzp_b200.EXPORTS:
        assert hasattr(lib, s), s
    assert set(toposzp_b200.EXPORTS) <= set(declared_symbols())


def test_version_string_without_gpu(libpath):
    lib = ctypes.CDLL(libpath)
    lib.szp_b200_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.szp_b200_version()


def test_batch_reserve_checks_its_arguments_without_gpu(libpath):
    """szp_b200_batch_reserve validates on the host before any device call."""
    import toposzp_b200 as T
    L = T.lib()
    assert L.szp_b200_batch_reserve(None, 4, 1 << 20) == -1
    assert "invalid arguments" in T.last_error()
