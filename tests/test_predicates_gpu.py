"""The device predicates -- FP32 stage, FP64 filter, exact expansion stage and
SoS, as the insertion rounds evaluate them -- against the oracle's exact
predicates (src/predicates.rs:106-217 orient3d_sos, 450-675 orient4d) on
records built to sit on every boundary between the stages: random points,
near-coplanar and near-cospherical sets a rounding away from degenerate, exact
lattice sets (SoS decides), tiny clusters whose permanents fall below the
FP32 stage's underflow guard, and the reference's super-vertex coordinates
(src/gpu/mod.rs:151-158).  Exactly degenerate sets are decided by the
modular exact stage (residues mod 2^64 and 2^61 - 1), near misses by its
Chinese-remainder sign or by the expansion stage when its bound does not
hold."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SUPER = np.array([[-100, -100, -100], [400, -100, -100], [-100, 400, -100], [-100, -100, 400]], np.float32)


def records(seed=7):
    r = np.random.default_rng(seed)
    out = []
    n = 3000
    out.append(r.random((n, 5, 3)).astype(np.float32))  # general position
    # near-coplanar: d in the plane of a, b, c up to the f32 rounding of d
    abc = r.random((n, 3, 3))
    uv = r.random((n, 2))
    d = abc[:, 0] + uv[:, :1] * (abc[:, 1] - abc[:, 0]) + uv[:, 1:] * (abc[:, 2] - abc[:, 0])
    out.append(np.concatenate([abc, d[:, None], r.random((n, 1, 3))], 1).astype(np.float32))
    # near-cospherical: five points on one sphere, rounded to f32
    c = r.random((n, 1, 3))
    rad = 0.05 + 0.4 * r.random((n, 1, 1))
    g = r.standard_normal((n, 5, 3))
    out.append((c + rad * g / np.linalg.norm(g, axis=2, keepdims=True)).astype(np.float32))
    # exact lattice picks: coplanar and cospherical sets, SoS decides
    lat = (r.integers(0, 4, (n, 5, 3)) / np.float32(4)).astype(np.float32)
    out.append(lat)
    # the 128^3 benchmark lattice (f32(i / 127), not dyadic): corners of
    # random boxes are exactly cospherical, faces exactly coplanar; the
    # modular exact stage decides these (and CRT signs of near misses)
    lo = r.integers(0, 120, (n, 1, 3))
    ext = r.integers(1, 8, (n, 1, 3))
    corner = r.integers(0, 2, (n, 5, 3))
    box = ((lo + corner * ext).astype(np.float64) / 127.0).astype(np.float32)
    out.append(box)
    out.append((r.integers(0, 128, (n, 5, 3)).astype(np.float64) / 127.0).astype(np.float32))
    # tiny clusters: permanents below the FP32 stage's guard
    base = r.random((n // 2, 1, 3))
    out.append((base + 1e-7 * r.random((n // 2, 5, 3))).astype(np.float32))
    out.append((1e-9 * r.random((n // 2, 5, 3))).astype(np.float32))
    # super vertices with real points
    mix = r.random((n, 5, 3)).astype(np.float32)
    for i in range(n):
        k = r.integers(1, 4)
        idx = r.choice(5, k, replace=False)
        mix[i, idx] = SUPER[r.choice(4, k, replace=False)]
    out.append(mix)
    pts = np.concatenate(out).astype(np.float32)
    keys = np.stack([r.permutation(5) + 5 * r.integers(0, 1000) for _ in range(len(pts))]).astype(np.uint32)
    return pts, keys


def test_device_predicates_match_oracle(gpu, oracle_mod):
    pts, keys = records()
    o3, o4 = gpu._core.predicate_signs(pts, keys)
    want3 = np.empty(len(pts), np.int32)
    want4 = np.empty(len(pts), np.int32)
    zero3 = zero4 = 0
    for i, (p, k) in enumerate(zip(pts.astype(np.float64), keys)):
        k = [int(x) for x in k]
        want3[i] = oracle_mod.orient3d_sos(p[0], p[1], p[2], p[3], *k[:4])
        want4[i] = oracle_mod.orient4d(p[0], p[1], p[2], p[3], p[4], *k)
        zero3 += oracle_mod.orient3d(p[0], p[1], p[2], p[3]) == 0
        zero4 += oracle_mod.insphere(p[0], p[1], p[2], p[3], p[4]) == 0
    assert zero3 > 100 and zero4 > 100  # SoS really decides some of them
    bad3 = np.nonzero(o3 != want3)[0]
    bad4 = np.nonzero(o4 != want4)[0]
    assert bad3.size == 0, (bad3[:10], pts[bad3[:3]])
    assert bad4.size == 0, (bad4[:10], pts[bad4[:3]])
