"""The C-ABI library builds, loads without a GPU, and exports exactly what
include/simplefmm_b200.h declares."""
import ctypes as C
import re
from pathlib import Path

import pytest

import simplefmm_b200 as sf
from simplefmm_b200 import build as B

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "simplefmm_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fmm_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    B.build()
    return sf.load_library()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_status_strings_and_version(lib):
    assert lib.fmm_status_string(0) == b"ok"
    assert lib.fmm_status_string(5) == b"degenerate input"
    assert lib.fmm_version().decode().count(".") == 2


def test_null_arguments_are_rejected_without_a_device(lib):
    h = C.c_void_p()
    assert lib.fmm_tree_build(None, None, 10, 0, 20, 64, 2, 0.0, C.byref(h)) == 1
    assert b"NULL" in lib.fmm_last_error()
    assert lib.fmm_plan_create(None, 8, 1, 0, C.byref(h)) == 1
    d = C.c_int()
    assert lib.fmm_tree_depth(None, C.byref(d)) == 1


def test_compiled_for_sm100a_only():
    assert B.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
