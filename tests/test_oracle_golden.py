"""Pins the oracle against the reference's own golden vectors and
known-answer tests (paths inside half-potato/wtet), and its predicates
against exact rational arithmetic.  CPU only."""
from fractions import Fraction
import itertools

import numpy as np
import pytest


# ---- Morton codes: src/morton.rs:88-151 -------------------------------------

def test_expand_bits_golden(oracle_mod):
    assert [oracle_mod.expand_bits(v) for v in (0, 1, 2, 4)] == [0, 1, 8, 64]


def test_interleave_golden(oracle_mod):
    assert oracle_mod.interleave_bits(1, 0, 0) == 1
    assert oracle_mod.interleave_bits(0, 1, 0) == 2
    assert oracle_mod.interleave_bits(0, 0, 1) == 4
    assert oracle_mod.interleave_bits(1, 1, 1) == 7


def test_morton_corners(oracle_mod):
    mn, mx = [0, 0, 0], [1, 1, 1]
    assert oracle_mod.morton_code([0, 0, 0], mn, mx) == 0
    assert oracle_mod.morton_code([1, 1, 1], mn, mx) == 0x3FFFFFFF
    assert oracle_mod.morton_code([0.5, 0.5, 0.5], mn, mx) == oracle_mod.morton_code([0.5, 0.5, 0.5], mn, mx)


def test_morton_order_is_stable(oracle_mod):
    pts = np.array([[0.5, 0.5, 0.5]] * 4 + [[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]], np.float32)
    order = oracle_mod.morton_order(pts)
    assert list(order) == [4, 0, 1, 2, 3, 5]


# ---- stride table and stratified order: src/gpu/mod.rs:607-696 --------------

@pytest.mark.parametrize("n,stride", [(100, 64), (1_000, 64), (10_000, 128), (100_000, 512), (1_000_000, 2048),
                                      (2_000_000, 4096), (10, 64), (1_000_000_000, 16384)])
def test_initial_stride_table(oracle_mod, n, stride):
    assert oracle_mod.initial_stride(n) == stride


def test_first_pass_small(oracle_mod):
    assert 2_000_000 // oracle_mod.initial_stride(2_000_000) < 1000


def test_stratified_pattern(oracle_mod):
    assert list(oracle_mod.strided_order(16, 8)) == [0, 8, 4, 12, 2, 6, 10, 14, 1, 3, 5, 7, 9, 11, 13, 15]


def test_stratified_preserves_count(oracle_mod):
    o = oracle_mod.strided_order(100, 64)
    assert sorted(o.tolist()) == list(range(100))


def test_stratified_order_prefix(oracle_mod):
    o = oracle_mod.strided_order(256, 128).tolist()
    assert o[:4] == [0, 128, 64, 192]


# ---- normalisation: src/tests.rs:132-155, bit-exact f32 ----------------------

def test_normalize_range(oracle_mod):
    pts = np.array([[10, 20, 30], [15, 25, 35], [12, 22, 32]], np.float32)
    out, mn, sc = oracle_mod.normalize(pts)
    assert out.min() >= 0 and out.max() <= 1
    assert abs(float(out.min())) < 1e-6 and abs(float(out.max()) - 1) < 1e-6


def test_normalize_bit_exact(oracle_mod):
    rng = np.random.default_rng(5)
    pts = (rng.standard_normal((1000, 3)) * 3 + 7).astype(np.float32)
    out, _, _ = oracle_mod.normalize(pts)
    mn = pts.min(0)
    ext = pts.max(0) - mn
    s = np.float32(max(float(ext.max()), 1e-10))
    ref = ((pts - mn) / s).astype(np.float32)
    assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))


# ---- predicate known answers: src/predicates.rs:690-820, src/tests.rs:12-80,1212-1281

def test_orient3d_signs(oracle_mod):
    assert oracle_mod.orient3d([0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]) < 0
    assert oracle_mod.orient3d([0, 0, 0], [0, 1, 0], [1, 0, 0], [0, 0, 1]) > 0
    assert oracle_mod.orient3d([0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]) == 0
    assert oracle_mod.orient3d([0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1e-12]) != 0
    assert oracle_mod.orient3d([0, 0, 0], [1, 0, 0], [0, 1, 0], [0.5, 0.5, 0]) == 0


def test_insphere_signs(oracle_mod):
    a, b, c, d = [1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]
    o = oracle_mod.orient3d(a, b, c, d)
    for e, inside in (([0, 0, 0], True), ([10, 10, 10], False), ([3 ** 0.5 - 1e-8, 0, 0], True)):
        s = oracle_mod.insphere(a, b, c, d, e)
        assert ((s > 0) if o > 0 else (s < 0)) == inside
    assert oracle_mod.insphere(a, b, c, d, [0, 0, 0]) * oracle_mod.insphere(a, c, b, d, [0, 0, 0]) < 0


def test_sos_known_answers(oracle_mod):
    a, b, c, d = [0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]
    r1 = oracle_mod.orient3d_sos(a, b, c, d, 0, 1, 2, 3)
    assert r1 != 0
    assert oracle_mod.orient3d_sos(b, a, c, d, 1, 0, 2, 3) == -r1
    nd = [0, 0, 1]
    raw = oracle_mod.orient3d(a, b, c, nd)
    assert oracle_mod.orient3d_sos(a, b, c, nd, 0, 1, 2, 3) == (1 if raw < 0 else -1)
    cs = ([1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1])
    assert oracle_mod.insphere(*cs) == 0
    assert oracle_mod.orient4d(*cs, 0, 1, 2, 3, 4) != 0
    t = ([1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1], [0, 0, 0])
    assert oracle_mod.orient4d(*t, 0, 1, 2, 3, 4) == np.sign(oracle_mod.insphere(*t))


# ---- exactness against rational arithmetic ----------------------------------

def det(m):
    m = [list(r) for r in m]
    n = len(m)
    s = Fraction(1)
    for i in range(n):
        piv = next((r for r in range(i, n) if m[r][i] != 0), None)
        if piv is None:
            return Fraction(0)
        if piv != i:
            m[i], m[piv] = m[piv], m[i]
            s = -s
        for r in range(i + 1, n):
            f = m[r][i] / m[i][i]
            for k in range(i, n):
                m[r][k] -= f * m[i][k]
        s *= m[i][i]
    return s


def F(p):
    return [Fraction(float(x)) for x in p]


def exact_orient3d(a, b, c, d):
    A, B, C, D = map(F, (a, b, c, d))
    return det([[A[i] - D[i] for i in range(3)], [B[i] - D[i] for i in range(3)], [C[i] - D[i] for i in range(3)]])


def exact_insphere(a, b, c, d, e):
    rows = []
    E = F(e)
    for p in (a, b, c, d):
        P = F(p)
        q = [P[i] - E[i] for i in range(3)]
        rows.append(q + [q[0] ** 2 + q[1] ** 2 + q[2] ** 2])
    return det(rows)


def sgn(x):
    return (x > 0) - (x < 0)


def near_degenerate_sets(rng, count):
    """Random f32 points, snapped lattice points and nearly coplanar / cospherical sets."""
    out = []
    for _ in range(count):
        kind = rng.integers(0, 4)
        if kind == 0:
            p = rng.random((5, 3)).astype(np.float32)
        elif kind == 1:
            p = (rng.integers(0, 4, (5, 3)) / np.float32(3)).astype(np.float32)
        elif kind == 2:
            p = rng.random((5, 3)).astype(np.float32)
            p[:, 2] = np.float32(0.25) + np.float32(1e-7) * rng.integers(-2, 3, 5).astype(np.float32)
        else:
            d = rng.standard_normal((5, 3))
            p = (0.5 + 0.25 * d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        out.append([list(map(float, q)) for q in p])
    return out


def test_orient3d_exact_vs_rational(oracle_mod):
    rng = np.random.default_rng(11)
    for pts in near_degenerate_sets(rng, 400):
        assert oracle_mod.orient3d(*pts[:4]) == sgn(exact_orient3d(*pts[:4]))


def test_insphere_exact_vs_rational(oracle_mod):
    rng = np.random.default_rng(12)
    for pts in near_degenerate_sets(rng, 300):
        assert oracle_mod.insphere(*pts) == sgn(exact_insphere(*pts))


def coplanar_sets(rng, count):
    """Quadruples (plus a fifth point) whose first four are exactly coplanar:
    the only case in which the SoS cascade evaluates the lifted orient3d
    (src/predicates.rs:513-556); there the reference's filtered form
    det[du, dv, |p - d|^2] equals det[u, v, |p|^2, 1]."""
    out = []
    for _ in range(count):
        kind = rng.integers(0, 3)
        if kind == 0:  # axis-aligned plane
            p = rng.random((5, 3)).astype(np.float32)
            ax = rng.integers(0, 3)
            p[:4, ax] = p[0, ax]
        elif kind == 1:  # lattice points on a lattice plane
            p = (rng.integers(0, 4, (5, 3)) / np.float32(3)).astype(np.float32)
            p[:4, 2] = p[0, 2]
        else:  # four corners of a box face (cospherical and coplanar)
            lo = rng.random(3).astype(np.float32)
            hi = (lo + rng.random(3).astype(np.float32)).astype(np.float32)
            p = np.array([[lo[0], lo[1], lo[2]], [hi[0], lo[1], lo[2]], [lo[0], hi[1], lo[2]],
                          [hi[0], hi[1], lo[2]], [lo[0], lo[1], hi[2]]], np.float32)
        out.append([list(map(float, q)) for q in p])
    return out


def test_lifted_helpers_vs_rational(oracle_mod):
    rng = np.random.default_rng(13)
    sets = coplanar_sets(rng, 200)
    for pts in sets:
        P = [F(p) for p in pts]
        w = [p[0] ** 2 + p[1] ** 2 + p[2] ** 2 for p in P]
        assert oracle_mod.orient3d(*pts[:4]) == 0
        for perm in ((0, 1, 2), (0, 2, 1), (1, 2, 0)):
            m = [[P[i][perm[0]], P[i][perm[1]], w[i], 1] for i in range(4)]
            assert oracle_mod.orient3d_lifted(*pts[:4], perm=perm) == sgn(det(m))
    for pts in near_degenerate_sets(rng, 200) + sets:
        P = [F(p) for p in pts]
        w = [p[0] ** 2 + p[1] ** 2 + p[2] ** 2 for p in P]
        for u in range(3):
            m = [[P[i][u], w[i], 1] for i in range(3)]
            assert oracle_mod.orient2d_lifted(*pts[:3], p0=u) == sgn(det(m))
        assert oracle_mod.orient1d_lifted(pts[0], pts[1]) == sgn(w[0] - w[1])


def test_sos_antisymmetry(oracle_mod):
    """Swapping two rows (with their indices) flips both SoS predicates."""
    rng = np.random.default_rng(14)
    for pts in near_degenerate_sets(rng, 150):
        idx = list(rng.permutation(50)[:5])
        r = oracle_mod.orient3d_sos(*pts[:4], *idx[:4])
        assert r in (-1, 1)
        for i, j in itertools.combinations(range(4), 2):
            q, k = list(pts[:4]), list(idx[:4])
            q[i], q[j] = q[j], q[i]
            k[i], k[j] = k[j], k[i]
            assert oracle_mod.orient3d_sos(*q, *k) == -r
        s = oracle_mod.orient4d(*pts, *idx)
        assert s in (-1, 1)
        q, k = list(pts), list(idx)
        q[0], q[1] = q[1], q[0]
        k[0], k[1] = k[1], k[0]
        assert oracle_mod.orient4d(*q, *k) == -s
