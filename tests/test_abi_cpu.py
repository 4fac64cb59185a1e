"""The C ABI library loads and exports every function include/ovx_fdg.h
declares; argument checks that need no GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import ovx_fdg_abi as abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "ovx_fdg.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ovx_\w+)\s*\(", text)))


def test_header_declares_functions():
    names = declared()
    assert "ovx_fdg_begin" in names and "ovx_fdg_finish" in names and "ovx_fdg_occupancy_noalloc" in names


def test_library_exports_every_declared_function():
    lib = abi.lib()
    for name in declared():
        assert hasattr(lib, name), name


def test_ctypes_prototypes_cover_the_header():
    assert sorted(n for n, _, _ in abi.PROTOTYPES) == declared()


def test_status_strings():
    lib = abi.lib()
    for code, text in [(0, b"ok"), (2, b"face index out of range"), (5, b"input or result too large")]:
        assert lib.ovx_fdg_status_string(code) == text
    assert lib.ovx_fdg_status_string(99) == b"unknown status"


def test_context_create_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert abi.lib().ovx_fdg_context_create(0, ctypes.byref(h)) == 1
    assert not h.value


def test_noalloc_argument_checks_need_no_gpu():
    lib = abi.lib()
    n = ctypes.c_int64(-1)
    g = abi.make_grid([1.0 / 512] * 3, [0, 0, 0, 512, 512, 512])
    # 64^3 bricks exceed the fixed scratch: rejected before any device work
    assert lib.ovx_fdg_occupancy_noalloc(None, None, 0, ctypes.byref(g), None, 0, ctypes.byref(n)) == 5
    bad = abi.make_grid([0.0, 0.1, 0.1], [0, 0, 0, 8, 8, 8])
    assert lib.ovx_fdg_occupancy_noalloc(None, None, 0, ctypes.byref(bad), None, 0, ctypes.byref(n)) == 1
    assert lib.ovx_fdg_occupancy_noalloc(None, None, 0, ctypes.byref(g), None, 0, None) == 1
