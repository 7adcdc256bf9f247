"""The C-ABI library loads and exports every entry point include/fasttree_b200.h declares (CPU).

No compute call is made here (no GPU is needed); the declarations are read from the header
so the check follows it.
"""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fasttree_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ft_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("ft_build_bvh", "ft_self_knn", "ft_knn", "ft_range", "ft_build_tree", "ft_sfc_encode",
              "ft_compute_bbox", "ft_tree_create", "ft_tree_destroy", "ft_context_create", "ft_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    from fasttree_b200 import capi
    lib = capi.lib()
    for s in declared_symbols():
        assert hasattr(lib, s), f"{s} declared in the header but not exported"
    assert set(capi.EXPORTED) == set(declared_symbols())


def test_version_and_error_string_without_gpu():
    from fasttree_b200 import capi
    lib = capi.lib()
    assert lib.ft_version() >= 10000
    assert isinstance(lib.ft_last_error(), bytes)


def test_invalid_options_rejected_before_any_device_work():
    from fasttree_b200 import capi
    lib = capi.lib()
    h = ctypes.c_void_p()
    o = capi.FtOptions(capi.U64, capi.MORTON, 0, 0, 0)  # Morton needs floating-point coordinates
    assert lib.ft_context_create(ctypes.byref(o), 0, ctypes.byref(h)) == capi.FT_ERR_INVALID_ARGUMENT
    o = capi.FtOptions(7, capi.MORTON, 0, 0, 0)
    assert lib.ft_context_create(ctypes.byref(o), 0, ctypes.byref(h)) == capi.FT_ERR_INVALID_ARGUMENT


def test_null_arguments_rejected():
    from fasttree_b200 import capi
    lib = capi.lib()
    assert lib.ft_context_create(None, 0, None) == capi.FT_ERR_INVALID_ARGUMENT
    assert lib.ft_tree_destroy(None, None) == capi.FT_OK
