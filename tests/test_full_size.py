"""Oracle parity at the benchmark sizes.

Each configuration is triangulated on the device, put in canonical form on
the device (wtet_canonicalize_device) and compared byte for byte, through
SHA-256, with the oracle's canonical output for the same seeded cloud
(tests/golden/full_size.json, written by tests/golden/make_full_size.py: the
oracle's sequential exact Bowyer-Watson, src/phase2.rs:383-606 semantics).
The output also passes the every-face exact verification
(wtet_verify_device: every face between finite tets, super-vertex faces
included, orientation of every tet, symmetric face-sharing links, the super
tetrahedron as the only hull).  The 1M unit sphere is additionally compared
with a live oracle run, and the device canonicaliser with the oracle's.

Sizes: 128^3 lattice (2,097,152 points), 1M unit sphere, 8M mixture seed 3
(the bench's cloud), 8M mixture seeds 101-105 with the plain and the learned
scheduler, 100k uniform, and all 4,096 clouds of the batched configuration.
"""
import json
import os

import numpy as np
import pytest

import fixtures as fx

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "full_size.json")) as _f:
    GOLDEN = json.load(_f)


def points_for(name):
    if name == "uniform100k":
        return fx.uniform(100_000, 1)
    if name == "lattice128":
        return fx.lattice(128)
    if name == "unit_sphere1M":
        return fx.unit_sphere(1_000_000, 2)
    if name.startswith("mixture8M_s"):
        return fx.mixture(8_000_000, int(name[len("mixture8M_s"):]))
    raise KeyError(name)


def run_and_digest(gpu, pts, vote="plain"):
    """Device triangulation -> device verification -> device canonical form ->
    SHA-256; returns (digest, canonical row count, verify report, stats)."""
    import torch

    d_pts = torch.from_numpy(pts).cuda()
    t, a = gpu.delaunay_device(d_pts, gpu.Config(vote=vote))
    rep = gpu.verify_device(d_pts, t, a)
    ct, ca = gpu.canonical_device(t, a, len(pts))
    dig = gpu.canonical_digest(ct, ca)
    rows = int(ct.shape[0])
    del t, a, ct, ca, d_pts
    torch.cuda.empty_cache()
    return dig, rows, rep


def assert_complete(rep, n):
    assert rep["violations"] == 0, rep
    assert rep["misoriented"] == 0, rep
    assert rep["broken_links"] == 0, rep
    assert rep["bad_vertex_ids"] == 0, rep
    assert rep["hull_faces"] == 4, rep
    # every interior face of T finite tets bounded by the super tetrahedron's 4
    # faces is shared by two tets: 4T = 2F + 4
    assert 4 * rep["finite_tets"] == 2 * rep["faces_checked"] + 4, rep


SINGLE = ["uniform100k", "lattice128", "unit_sphere1M", "mixture8M_s3"]


@pytest.mark.parametrize("name", SINGLE)
def test_full_size_matches_oracle(gpu, name):
    pts = points_for(name)
    want = GOLDEN[name]
    dig, rows, rep = run_and_digest(gpu, pts)
    assert_complete(rep, len(pts))
    assert rows == want["canonical_rows"], (rows, want)
    assert dig == want["sha256"], f"{name}: canonical tets/adjacency differ from the oracle's"


@pytest.mark.parametrize("seed", [101, 102, 103, 104, 105])
@pytest.mark.parametrize("vote", ["plain", "learned"])
def test_learned_config_matches_oracle(gpu, seed, vote):
    """The learned-vote configuration: 8M mixture clouds from seeds 101-105,
    with either scheduler, give the oracle's tet set and adjacency."""
    name = f"mixture8M_s{seed}"
    pts = points_for(name)
    dig, rows, rep = run_and_digest(gpu, pts, vote)
    assert_complete(rep, len(pts))
    assert rows == GOLDEN[name]["canonical_rows"]
    assert dig == GOLDEN[name]["sha256"], f"{name} ({vote}): differs from the oracle"


def test_sphere_live_oracle(gpu, oracle_mod):
    """1M unit sphere against an oracle run in the same process (not only the
    stored digest), compared as arrays; the device canonical form equals the
    oracle's canonicaliser applied to the device output."""
    pts = fx.unit_sphere(1_000_000, 2)
    r = gpu.delaunay(pts)
    tets, adj, st = oracle_mod.delaunay(pts, 1)
    ot, oa = oracle_mod.canonical(tets, adj, len(pts))
    gt, ga = gpu.canonical(r.tets, r.adjacency, len(pts))
    assert np.array_equal(gt, ot) and np.array_equal(ga, oa)
    ht, ha = oracle_mod.canonical(r.tets, r.adjacency, len(pts))
    assert np.array_equal(gt, ht) and np.array_equal(ga, ha)
    assert oracle_mod.digest(ot, oa) == GOLDEN["unit_sphere1M"]["sha256"]


def test_full_size_batched_matches_oracle(gpu, oracle_mod):
    """All 4,096 clouds of the batched configuration (log-uniform sizes in
    [64, 65536], about 40M points): every cloud's canonical output equals the
    oracle's triangulation of that cloud alone."""
    g = np.load(os.path.join(HERE, "golden", "batched_digests.npz"))
    clouds = fx.batched_clouds(4096, 4)
    assert np.array_equal(np.array([len(c) for c in clouds]), g["sizes"])
    res = gpu.delaunay_batched(clouds)
    bad = []
    for i, (pts, r) in enumerate(zip(clouds, res)):
        ct, ca = oracle_mod.canonical(r.tets, r.adjacency, len(pts))
        if bytes.fromhex(oracle_mod.digest(ct, ca)) != g["digests"][i].tobytes():
            bad.append(i)
    assert not bad, f"{len(bad)} clouds differ from the oracle, first {bad[:10]}"


def test_verify_catches_planted_mistakes(gpu):
    """The every-face check sees a swapped vertex (non-Delaunay faces and
    broken links), a flipped tet and a broken link, including on tets that
    touch the super vertices (which the reference-compatible check skips)."""
    pts = fx.uniform(20000, 5)
    n = len(pts)
    r = gpu.delaunay(pts)
    rep = gpu.verify(pts, r)
    assert_complete(rep, n)
    t = r.tets.copy()
    # a tet with a super vertex and no infinity vertex
    sup = np.nonzero(((t >= n) & (t < n + 4)).any(axis=1) & ~(t == n + 4).any(axis=1))[0]
    k = int(sup[0])
    t[k, [0, 1]] = t[k, [1, 0]]  # flips its orientation
    rep = gpu.verify(pts, gpu.DelaunayResult(t, r.adjacency, r.failed_verts))
    assert rep["misoriented"] == 1
    a = r.adjacency.copy()
    a[k, 0] = a[k, 1]  # a link that is no longer symmetric
    rep = gpu.verify(pts, gpu.DelaunayResult(r.tets, a, r.failed_verts))
    assert rep["broken_links"] >= 1
    assert gpu.check_quality(pts, gpu.DelaunayResult(r.tets, r.adjacency, r.failed_verts))[0] == 0
