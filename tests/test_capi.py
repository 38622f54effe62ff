"""C ABI and host-side API checks that need no GPU: libwtet.so loads, exports
every entry point include/wtet.h declares, and the Python mirror of wtet._core
validates input exactly like the reference (python/tests/test_basic.py,
src/python.rs:166-402)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if name.endswith(".h"):
            text = open(os.path.join(ROOT, "include", name)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            syms |= set(re.findall(r"\b(wtet_[a-z0-9_]+)\s*\(", text))
    return syms


def test_library_exports_every_declared_symbol(wt):
    lib = ctypes.CDLL(wt._core.lib_path())
    syms = declared_symbols()
    assert "wtet_delaunay" in syms and "wtet_check_quality" in syms
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing


def test_config_defaults_match_reference(wt):
    c = wt._core._Config()
    wt._core.load().wtet_config_default(ctypes.byref(c))
    # GDelConfig::default(), src/types.rs:49-61
    assert (c.insertion_rule, c.enable_flipping, c.enable_sorting, c.enable_hilbert_sorting, c.enable_splaying,
            c.max_insert_iterations, c.max_flip_iterations) == (0, 1, 0, 0, 1, 100, 10)


def test_invalid_insertion_rule(wt):
    with pytest.raises(ValueError, match="Invalid insertion_rule"):
        wt.Config(insertion_rule="invalid")
    with pytest.raises(ValueError, match="Invalid insertion_rule"):
        wt.Config(insertion_rule="midpoint")


def test_config_repr(wt):
    r = repr(wt.Config(insertion_rule="circumcenter", enable_flipping=True))
    assert "Config" in r and "circumcenter" in r and "flipping=True" in r


def test_invalid_shapes(wt):
    with pytest.raises(ValueError, match="must have shape"):
        wt.delaunay(np.array([1, 2, 3], np.float32))
    with pytest.raises(ValueError, match="must have shape"):
        wt.delaunay(np.array([[1, 2], [3, 4]], np.float32))


def test_too_few_points(wt):
    with pytest.raises(ValueError, match="at least 4 points"):
        wt.delaunay(np.array([[0, 0, 0], [1, 0, 0]], np.float32))


def test_c_abi_rejects_small_input(wt):
    L = wt._core.load()
    pts = np.zeros((3, 3), np.float32)
    m = ctypes.c_uint64(0)
    rc = L.wtet_delaunay_into(ctypes.c_void_p(pts.ctypes.data), 3, None, None, None, 0, ctypes.byref(m), None, None)
    assert rc == wt._core.WTET_ERR_ARG
    assert b"at least 4 points" in L.wtet_last_error()


def test_encode_decode_adjacency(wt):
    assert wt.decode_adjacency(wt.encode_adjacency(42, 2)) == (42, 2)
    assert wt.decode_adjacency(wt.encode_adjacency(0, 0)) == (0, 0)
    mx = (1 << 27) - 1
    for f in range(4):
        assert wt.decode_adjacency(wt.encode_adjacency(mx, f)) == (mx, f)


def test_invalid_constant(wt):
    assert wt.INVALID == 2 ** 32 - 1
    assert wt.__version__


def test_result_repr(wt):
    r = wt.DelaunayResult(np.zeros((5, 4), np.uint32), np.zeros((5, 4), np.uint32), np.zeros(0, np.uint32))
    assert repr(r) == "DelaunayResult(num_tets=5, failed_verts=0)"
