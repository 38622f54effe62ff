"""The modular exact stage of the device predicates (exact.cuh:
orient3d_modular, insphere_modular), restated on the CPU with Python
integers: every coordinate is an integer multiple of 2^S, the determinant is
evaluated on residues mod 2^64 and mod the Mersenne prime 2^61 - 1, and the
Chinese remainder theorem gives the exact value whenever the FP64 filter's
bound puts it below 2^122.  Checked against exact rational determinants on
random, near-degenerate and exactly degenerate records (boxes of the 128^3
benchmark lattice, whose corners are cospherical).  The device code itself is
checked against the oracle by tests/test_predicates_gpu.py."""
import math
from fractions import Fraction

import numpy as np

P61 = (1 << 61) - 1
M64 = 1 << 64
EPS = 2.0 ** -53
ISP_BOUND = (16.0 + 224.0 * EPS) * EPS
O3D_BOUND = (7.0 + 56.0 * EPS) * EPS


def dyadic(x):
    """x = (-1)^neg m 2^e with m odd, or m = 0."""
    if x == 0:
        return 0, None, False
    m, e = math.frexp(abs(x))  # |x| = m 2^e, 0.5 <= m < 1
    mi = int(m * 2 ** 53)
    e -= 53
    while mi % 2 == 0:
        mi //= 2
        e += 1
    return mi, e, x < 0


def residues(vals):
    parts = [dyadic(v) for v in vals]
    S = min(e for m, e, _ in parts if m)
    out = []
    for m, e, neg in parts:
        if not m:
            out.append((0, 0))
            continue
        k = e - S
        a = (m << k) % M64 if k < 64 else 0
        b = (m * pow(2, k % 61, P61)) % P61
        out.append(((-a) % M64, (-b) % P61) if neg else (a, b))
    return S, out


def crt_sign(a, b):
    k = ((b - a % P61) * (1 << 58)) % P61  # 1/8 = 2^58 mod P, 2^64 = 8 mod P
    x = a + (k << 64)
    if x == 0:
        return 0
    return -1 if x >= (P61 << 63) else 1


class R:
    """A value mod 2^64 and mod P61 (the device's Res)."""

    def __init__(self, a, b):
        self.a, self.b = a % M64, b % P61

    def __add__(self, o):
        return R(self.a + o.a, self.b + o.b)

    def __sub__(self, o):
        return R(self.a - o.a, self.b - o.b)

    def __mul__(self, o):
        return R(self.a * o.a, self.b * o.b)


def insphere_exact(p):
    q = [[Fraction(c) for c in pt] for pt in p]
    d = [[q[i][j] - q[4][j] for j in range(3)] for i in range(4)]
    rows = [[x, y, z, x * x + y * y + z * z] for x, y, z in d]
    return det4(rows)


def det4(m):
    def det3(a):
        return (a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0])
                + a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]))
    return sum((-1) ** c * m[0][c] * det3([row[:c] + row[c + 1:] for row in m[1:]]) for c in range(4))


def insphere_filter(p):
    """det and err of the FP64 filter, one rounding per operation (Python floats)."""
    ae = [[p[i][j] - p[4][j] for j in range(3)] for i in range(4)]
    (aex, aey, aez), (bex, bey, bez), (cex, cey, cez), (dex, dey, dez) = ae
    aexbey, bexaey = aex * bey, bex * aey
    bexcey, cexbey = bex * cey, cex * bey
    cexdey, dexcey = cex * dey, dex * cey
    dexaey, aexdey = dex * aey, aex * dey
    aexcey, cexaey = aex * cey, cex * aey
    bexdey, dexbey = bex * dey, dex * bey
    ab, bc, cd, da = aexbey - bexaey, bexcey - cexbey, cexdey - dexcey, dexaey - aexdey
    ac, bd = aexcey - cexaey, bexdey - dexbey
    abc = (aez * bc - bez * ac) + cez * ab
    bcd = (bez * cd - cez * bd) + dez * bc
    cda = (cez * da + dez * ac) + aez * cd
    dab = (dez * ab + aez * bd) + bez * da
    al = (aex * aex + aey * aey) + aez * aez
    bl = (bex * bex + bey * bey) + bez * bez
    cl = (cex * cex + cey * cey) + cez * cez
    dl = (dex * dex + dey * dey) + dez * dez
    det = (dl * abc - cl * dab) + (bl * cda - al * bcd)
    az, bz, cz, dz = abs(aez), abs(bez), abs(cez), abs(dez)
    p_ab, p_bc = abs(aexbey) + abs(bexaey), abs(bexcey) + abs(cexbey)
    p_cd, p_da = abs(cexdey) + abs(dexcey), abs(dexaey) + abs(aexdey)
    p_ac, p_bd = abs(aexcey) + abs(cexaey), abs(bexdey) + abs(dexbey)
    perm = (((((p_cd * bz + p_bd * cz) + p_bc * dz) * al + ((p_da * cz + p_ac * dz) + p_cd * az) * bl)
             + ((p_ab * dz + p_bd * az) + p_da * bz) * cl) + ((p_bc * az + p_ac * bz) + p_ab * cz) * dl)
    return det, ISP_BOUND * perm


def insphere_modular(p, err):
    """The device stage: exact sign, or None when it does not apply."""
    flat = [c for pt in p for c in pt]
    if all(c == 0 for c in flat):
        return 0
    S, res = residues(flat)
    if S < -160 or not (math.ldexp(err * (2.0 + 2.0 ** -39), -5 * S) < 2.0 ** 122):
        return None
    X = [R(a, b) for a, b in res]
    pts = [X[3 * i:3 * i + 3] for i in range(5)]
    d = [[pts[i][j] - pts[4][j] for j in range(3)] for i in range(4)]
    rows = [[x, y, z, x * x + y * y + z * z] for x, y, z in d]
    det = det4_ring(rows)
    return crt_sign(det.a, det.b)


def det4_ring(m):
    def det3(a):
        return (a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0])
                + a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]))
    out = R(0, 0)
    for c in range(4):
        t = m[0][c] * det3([row[:c] + row[c + 1:] for row in m[1:]])
        out = out + t if c % 2 == 0 else out - t
    return out


def records(seed=3, n=400):
    r = np.random.default_rng(seed)
    out = []
    lo = r.integers(0, 120, (n, 1, 3))
    ext = r.integers(1, 8, (n, 1, 3))
    corner = r.integers(0, 2, (n, 5, 3))
    out.append(((lo + corner * ext).astype(np.float64) / 127.0).astype(np.float32))  # cospherical boxes
    c = r.random((n, 1, 3))
    g = r.standard_normal((n, 5, 3))
    out.append((c + 0.2 * g / np.linalg.norm(g, axis=2, keepdims=True)).astype(np.float32))  # near misses
    out.append(r.random((n, 5, 3)).astype(np.float32))
    sup = np.array([[-100, -100, -100], [400, -100, -100], [-100, 400, -100], [-100, -100, 400]], np.float32)
    box = out[0].copy()
    box[:, 0] = sup[r.integers(0, 4, n)]
    out.append(box)
    return np.concatenate(out).astype(np.float64)


def test_crt_reconstructs_signed_values():
    r = np.random.default_rng(1)
    for _ in range(2000):
        x = int(r.integers(-(1 << 62), 1 << 62)) * int(r.integers(1, 1 << 60))
        assert crt_sign(x % M64, x % P61) == (x > 0) - (x < 0)
    assert crt_sign(0, 0) == 0


def test_modular_insphere_is_exact_when_it_answers():
    answered = zeros = 0
    for p in records():
        pts = [list(map(float, q)) for q in p]
        exact = insphere_exact(pts)
        want = (exact > 0) - (exact < 0)
        det, err = insphere_filter(pts)
        assert abs(Fraction(det) - exact) <= Fraction(err)  # the filter's bound holds
        if det > err or -det > err:
            continue  # the filter decides; the stage never runs
        got = insphere_modular(pts, err)
        if got is None:
            continue
        answered += 1
        zeros += want == 0
        assert got == want, (pts, got, want)
    assert answered > 300 and zeros > 100  # cospherical lattice boxes reach it and are decided
