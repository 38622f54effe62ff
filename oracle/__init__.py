"""Oracle: a CPU restatement of the reference's exact Delaunay semantics.

Test infrastructure only.  tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py load it as the checker;
the wtet_b200 product never imports, links or calls it.

Restated reference behaviour (paths inside half-potato/wtet):
  * exact orient3d / insphere (src/predicates.rs:14-21, via geometry-predicates
    0.3.0 there, Shewchuk's published adaptive method here),
  * the SoS cascades orient3d_sos and orient4d (src/predicates.rs:106-675),
  * Bowyer-Watson over the normalised points plus four super vertices
    (src/phase2.rs:383-606, src/gpu/mod.rs:151-158, src/lib.rs:313-337),
  * Morton codes, Morton order, stride table and stratified order
    (src/morton.rs:22-80, src/gpu/mod.rs:422-600),
  * check_delaunay_quality (src/lib.rs:25-78).

Parity pin: predicates against exact rational arithmetic and the reference's
predicate known-answer tests; Morton / stride / stratified order against the
reference's golden vectors; triangulations against the reference's structural
and exact local-Delaunay validators.  No reference test pins an exact tet set
and the reference cannot be built here (no Rust toolchain, crates not vendored),
so the tet set itself rests on the uniqueness of the SoS Delaunay triangulation.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

INVALID = 0xFFFFFFFF


class OracleStats(ctypes.Structure):
    _fields_ = [
        ("num_tets", ctypes.c_uint64),
        ("cavity_tets", ctypes.c_uint64),
        ("boundary_faces", ctypes.c_uint64),
        ("max_cavity", ctypes.c_uint32),
        ("max_boundary", ctypes.c_uint32),
        ("walk_steps", ctypes.c_uint64),
        ("o3d_exact", ctypes.c_uint64),
        ("o3d_sos", ctypes.c_uint64),
        ("isp_exact", ctypes.c_uint64),
        ("isp_sos", ctypes.c_uint64),
        ("cavity_hist", ctypes.c_uint64 * 16),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["cavity_hist"] = list(self.cavity_hist)
        return d


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile beside this file (make skips the
    work when the library is newer than its sources)."""
    if force or not os.path.exists(_LIB_PATH) or _stale():
        subprocess.run(["make", "-s", "-C", _HERE] + (["-B"] if force else []), check=True)
    return _LIB_PATH


def _stale() -> bool:
    t = os.path.getmtime(_LIB_PATH)
    srcs = [f for f in os.listdir(_HERE) if f.endswith((".cpp", ".hpp", ".h"))]
    return any(os.path.getmtime(os.path.join(_HERE, f)) > t for f in srcs)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        d3 = ctypes.POINTER(ctypes.c_double)
        u32 = ctypes.c_uint32
        L.oracle_normalize.argtypes = [P, ctypes.c_uint64, P, P, P]
        L.oracle_expand_bits.restype = u32
        L.oracle_expand_bits.argtypes = [u32]
        L.oracle_interleave_bits.restype = u32
        L.oracle_interleave_bits.argtypes = [u32, u32, u32]
        L.oracle_morton_code.restype = u32
        L.oracle_morton_code.argtypes = [P, P, P]
        L.oracle_morton_order.argtypes = [P, ctypes.c_uint64, P]
        L.oracle_initial_stride.restype = ctypes.c_uint64
        L.oracle_initial_stride.argtypes = [ctypes.c_uint64]
        L.oracle_strided_order.argtypes = [ctypes.c_uint64, ctypes.c_uint64, P]
        L.oracle_orient3d.argtypes = [d3] * 4
        L.oracle_insphere.argtypes = [d3] * 5
        L.oracle_orient3d_sos.argtypes = [d3] * 4 + [u32] * 4
        L.oracle_orient4d.argtypes = [d3] * 5 + [u32] * 5
        L.oracle_orient3d_lifted.argtypes = [d3] * 4 + [ctypes.c_int] * 3
        L.oracle_orient2d_lifted.argtypes = [d3] * 3 + [ctypes.c_int]
        L.oracle_orient1d_lifted.argtypes = [d3] * 2
        L.oracle_dt_run.restype = P
        L.oracle_dt_run.argtypes = [P, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(OracleStats)]
        L.oracle_dt_num_tets.restype = ctypes.c_uint64
        L.oracle_dt_num_tets.argtypes = [P]
        L.oracle_dt_copy.argtypes = [P, P, P]
        L.oracle_dt_free.argtypes = [P]
        L.oracle_dt_num_failed.restype = ctypes.c_uint64
        L.oracle_dt_num_failed.argtypes = [P]
        L.oracle_dt_copy_failed.argtypes = [P, P]
        L.oracle_last_error.restype = ctypes.c_char_p
        for name in ("oracle_check_delaunay_quality", "oracle_check_local_delaunay"):
            f = getattr(L, name)
            f.restype = ctypes.c_int64
            f.argtypes = [P, ctypes.c_uint64, P, P, ctypes.c_uint64]
        L.oracle_canonical.restype = ctypes.c_uint64
        L.oracle_canonical.argtypes = [P, P, ctypes.c_uint64, ctypes.c_uint32, P, P]
        L.oracle_check_orientation.restype = ctypes.c_int64
        L.oracle_check_orientation.argtypes = [P, ctypes.c_uint64, P, ctypes.c_uint64]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f32(points) -> np.ndarray:
    return np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)


def _d3(p):
    a = (ctypes.c_double * 3)(*[float(v) for v in p])
    return a


def normalize(points):
    pts = _f32(points)
    out = np.empty_like(pts)
    mn = np.empty(3, np.float32)
    sc = np.empty(1, np.float32)
    lib().oracle_normalize(_ptr(pts), pts.shape[0], _ptr(out), _ptr(mn), _ptr(sc))
    return out, mn, float(sc[0])


def expand_bits(v: int) -> int:
    return int(lib().oracle_expand_bits(v))


def interleave_bits(x: int, y: int, z: int) -> int:
    return int(lib().oracle_interleave_bits(x, y, z))


def morton_code(p, mn, mx) -> int:
    a = np.asarray(p, np.float32)
    b = np.asarray(mn, np.float32)
    c = np.asarray(mx, np.float32)
    return int(lib().oracle_morton_code(_ptr(a), _ptr(b), _ptr(c)))


def morton_order(points) -> np.ndarray:
    pts = _f32(points)
    out = np.empty(pts.shape[0], np.uint32)
    lib().oracle_morton_order(_ptr(pts), pts.shape[0], _ptr(out))
    return out


def initial_stride(n: int) -> int:
    return int(lib().oracle_initial_stride(n))


def strided_order(n: int, stride: int) -> np.ndarray:
    out = np.empty(n, np.uint32)
    lib().oracle_strided_order(n, stride, _ptr(out))
    return out


def orient3d(a, b, c, d) -> int:
    return lib().oracle_orient3d(_d3(a), _d3(b), _d3(c), _d3(d))


def insphere(a, b, c, d, e) -> int:
    return lib().oracle_insphere(_d3(a), _d3(b), _d3(c), _d3(d), _d3(e))


def orient3d_sos(a, b, c, d, ia, ib, ic, id_) -> int:
    return lib().oracle_orient3d_sos(_d3(a), _d3(b), _d3(c), _d3(d), ia, ib, ic, id_)


def orient4d(a, b, c, d, e, ia, ib, ic, id_, ie) -> int:
    return lib().oracle_orient4d(_d3(a), _d3(b), _d3(c), _d3(d), _d3(e), ia, ib, ic, id_, ie)


def orient3d_lifted(a, b, c, d, perm=(0, 1, 2)) -> int:
    return lib().oracle_orient3d_lifted(_d3(a), _d3(b), _d3(c), _d3(d), *perm)


def orient2d_lifted(a, b, c, p0=0) -> int:
    return lib().oracle_orient2d_lifted(_d3(a), _d3(b), _d3(c), p0)


def orient1d_lifted(a, b) -> int:
    return lib().oracle_orient1d_lifted(_d3(a), _d3(b))


def delaunay(points, order_mode: int = 1):
    """Oracle triangulation: (tets (M,4) u32, adjacency (M,4) u32, stats dict).

    Vertex ids are original indices, super vertices n..n+3; adjacency is
    (tet << 5) | face with INVALID on the super tetrahedron's hull.  Exact
    duplicates (equal normalised coordinates) after the first occurrence are
    left out and listed in stats["failed"]."""
    pts = _f32(points)
    st = OracleStats()
    h = lib().oracle_dt_run(_ptr(pts), pts.shape[0], order_mode, ctypes.byref(st))
    if not h:
        raise RuntimeError("oracle: " + lib().oracle_last_error().decode())
    try:
        m = lib().oracle_dt_num_tets(h)
        tets = np.empty((m, 4), np.uint32)
        adj = np.empty((m, 4), np.uint32)
        lib().oracle_dt_copy(h, _ptr(tets), _ptr(adj))
        nf = lib().oracle_dt_num_failed(h)
        failed = np.empty(nf, np.uint32)
        lib().oracle_dt_copy_failed(h, _ptr(failed))
    finally:
        lib().oracle_dt_free(h)
    d = st.as_dict()
    d["failed"] = failed
    return tets, adj, d


def triangulate_count(points, order_mode: int = 1) -> int:
    """Runs the oracle triangulation and returns its tet count without
    copying the output out (for timing the CPU path: the run itself still
    builds the compacted output rows, as the reference's readback does)."""
    pts = _f32(points)
    st = OracleStats()
    h = lib().oracle_dt_run(_ptr(pts), pts.shape[0], order_mode, ctypes.byref(st))
    if not h:
        raise RuntimeError("oracle: " + lib().oracle_last_error().decode())
    try:
        return int(lib().oracle_dt_num_tets(h))
    finally:
        lib().oracle_dt_free(h)


def check_delaunay_quality(points, tets, adj) -> int:
    pts = _f32(points)
    t = np.ascontiguousarray(tets, np.uint32)
    a = np.ascontiguousarray(adj, np.uint32)
    return int(lib().oracle_check_delaunay_quality(_ptr(pts), pts.shape[0], _ptr(t), _ptr(a), t.shape[0]))


def check_local_delaunay(points, tets, adj) -> int:
    pts = _f32(points)
    t = np.ascontiguousarray(tets, np.uint32)
    a = np.ascontiguousarray(adj, np.uint32)
    return int(lib().oracle_check_local_delaunay(_ptr(pts), pts.shape[0], _ptr(t), _ptr(a), t.shape[0]))


def check_orientation(points, tets) -> int:
    pts = _f32(points)
    t = np.ascontiguousarray(tets, np.uint32)
    return int(lib().oracle_check_orientation(_ptr(pts), pts.shape[0], _ptr(t), t.shape[0]))


def canonical(tets, adj, n: int):
    """Canonical parity form (C++, canon.cpp); same result as canonical_numpy."""
    t = np.ascontiguousarray(tets, np.uint32).reshape(-1, 4)
    a = np.ascontiguousarray(adj, np.uint32).reshape(-1, 4)
    m = t.shape[0]
    ot = np.empty((m, 4), np.uint32)
    oa = np.empty((m, 4), np.uint32)
    k = int(lib().oracle_canonical(_ptr(t), _ptr(a), m, n, _ptr(ot), _ptr(oa)))
    ot.resize((k, 4), refcheck=False)
    oa.resize((k, 4), refcheck=False)
    return ot, oa


def digest(canon_tets, canon_adj) -> str:
    """SHA-256 of a canonical form: the tets' bytes, then the adjacency's
    (little-endian u32)."""
    import hashlib

    h = hashlib.sha256()
    h.update(np.ascontiguousarray(canon_tets, "<u4").tobytes())
    h.update(np.ascontiguousarray(canon_adj, "<u4").tobytes())
    return h.hexdigest()


def canonical_numpy(tets, adj, n: int):
    """Canonical parity form.

    T_all: every tet without the infinity vertex n+4, vertex ids sorted, rows
    sorted lexicographically.  Adjacency: for each canonical tet and each face
    opposite sorted slot f, (canonical index of the neighbour << 5) | slot of the
    opposite vertex in the neighbour's sorted row, or INVALID -- derived from
    the given adjacency links, so it also checks them."""
    tets = np.asarray(tets, np.uint32).reshape(-1, 4)
    adj = np.asarray(adj, np.uint32).reshape(-1, 4)
    inf = n + 4
    keep = ~(tets == inf).any(axis=1)
    order_in_row = np.argsort(tets, axis=1, kind="stable")
    srt = np.take_along_axis(tets, order_in_row, axis=1)
    kept_idx = np.nonzero(keep)[0]
    rows = srt[kept_idx]
    lex = np.lexsort((rows[:, 3], rows[:, 2], rows[:, 1], rows[:, 0]))
    canon_tets = rows[lex]
    # position of each original tet in canonical order (or -1)
    pos = np.full(tets.shape[0], -1, np.int64)
    pos[kept_idx[lex]] = np.arange(kept_idx.size)
    # slot of original face f in the sorted row: inverse of order_in_row
    inv = np.argsort(order_in_row, axis=1)
    canon_adj = np.full((kept_idx.size, 4), INVALID, np.uint32)
    src = kept_idx[lex]
    for f in range(4):
        a = adj[src, f]
        valid = a != INVALID
        nb = (a >> 5).astype(np.int64)
        nf = (a & 3).astype(np.int64)
        # face f of the original row corresponds to sorted slot inv[src, f]
        sslot = inv[src, f]
        nb_ok = valid & (nb < tets.shape[0])
        nbpos = np.where(nb_ok, pos[np.where(nb_ok, nb, 0)], -1)
        good = nb_ok & (nbpos >= 0)
        nslot = np.where(good, inv[np.where(nb_ok, nb, 0), nf], 0)
        val = np.where(good, (nbpos.astype(np.uint64) << 5) | nslot.astype(np.uint64), INVALID).astype(np.uint32)
        canon_adj[np.arange(src.size), sslot] = val
    return canon_tets, canon_adj
