"""Parity of the CUDA path with the oracle (the reference's exact semantics):
the canonical tet set and the canonical adjacency (derived from the GPU's own
links) must be byte-identical, on the committed golden fixtures, on seeded
cases of every benchmark distribution at sizes the oracle finishes in seconds,
and on the reference's own degenerate fixtures.  All calls go through the C
ABI (libwtet.so)."""
import os

import numpy as np
import pytest

import fixtures as fx
from validators import check_adjacency, euler, finite

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def assert_parity(wt, oracle_mod, pts, config=None):
    n = len(pts)
    r = wt.delaunay(pts, config)
    tets, adj, st = oracle_mod.delaunay(pts, 1)
    gt, ga = oracle_mod.canonical(r.tets, r.adjacency, n)
    ot, oa = oracle_mod.canonical(tets, adj, n)
    assert gt.shape == ot.shape, (gt.shape, ot.shape)
    assert np.array_equal(gt, ot), "tet sets differ"
    assert np.array_equal(ga, oa), "adjacency differs"
    assert np.array_equal(np.sort(r.failed_verts), st["failed"])
    # structure of the raw output: 4 infinity tets, symmetric links, oriented tets
    inf = (r.tets == n + 4).any(axis=1)
    assert inf.sum() == 4
    check_adjacency(r.tets, r.adjacency)
    assert oracle_mod.check_orientation(pts, r.tets) == 0
    return r


def test_golden_fixtures(gpu, oracle_mod):
    g = np.load(os.path.join(HERE, "golden", "golden.npz"))
    for name in g["names"]:
        pts = g[f"{name}/points"]
        r = gpu.delaunay(pts)
        ct, ca = oracle_mod.canonical(r.tets, r.adjacency, len(pts))
        assert np.array_equal(ct, g[f"{name}/tets"]), name
        assert np.array_equal(ca, g[f"{name}/adjacency"]), name


CASES = {
    "four": lambda: np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32),
    "cube": fx.cube,
    "icosahedron": fx.icosahedron,
    "grid4": lambda: fx.lattice(4),
    "grid5": lambda: fx.lattice(5),
    "grid12": lambda: fx.lattice(12),
    "lattice24": lambda: fx.lattice(24),
    "shell30": lambda: fx.sphere_shell(30, 42),
    "shell5k": lambda: fx.sphere_shell(5000, 7),
    "unit_sphere20k": lambda: fx.unit_sphere(20000, 2),
    "uniform100": lambda: fx.uniform(100, 42),
    "uniform100k": lambda: fx.uniform(100_000, 1),
    "clusters": lambda: fx.clustered(5000, 4, 9),
    "mixture50k": lambda: fx.mixture(50_000, 3),
    "coplanar_offset": fx.coplanar_with_offset,
    "near_collinear": fx.near_collinear,
    "duplicates": fx.with_duplicates,
    "scaled": lambda: (fx.uniform(2000, 5) * np.float32(1000) - np.float32(300)).astype(np.float32),
}


@pytest.mark.parametrize("name", list(CASES))
def test_parity(gpu, oracle_mod, name):
    assert_parity(gpu, oracle_mod, CASES[name]())


def test_insertion_rules_agree(gpu, oracle_mod):
    pts = fx.uniform(20000, 8)
    a = gpu.delaunay(pts, gpu.Config(insertion_rule="circumcenter"))
    b = gpu.delaunay(pts, gpu.Config(insertion_rule="centroid"))
    ca = oracle_mod.canonical(a.tets, a.adjacency, len(pts))
    cb = oracle_mod.canonical(b.tets, b.adjacency, len(pts))
    assert np.array_equal(ca[0], cb[0]) and np.array_equal(ca[1], cb[1])


def test_repeatable(gpu, oracle_mod):
    pts = fx.mixture(30000, 9)
    a = gpu.delaunay(pts)
    b = gpu.delaunay(pts)
    ca = oracle_mod.canonical(a.tets, a.adjacency, len(pts))
    cb = oracle_mod.canonical(b.tets, b.adjacency, len(pts))
    assert np.array_equal(ca[0], cb[0]) and np.array_equal(ca[1], cb[1])


def test_batched_matches_single(gpu, oracle_mod):
    clouds = fx.batched_clouds(24, 4, lo=64, hi=4096)
    res = gpu.delaunay_batched(clouds)
    assert len(res) == len(clouds)
    for pts, r in zip(clouds, res):
        tets, adj, st = oracle_mod.delaunay(pts, 1)
        gt, ga = oracle_mod.canonical(r.tets, r.adjacency, len(pts))
        ot, oa = oracle_mod.canonical(tets, adj, len(pts))
        assert np.array_equal(gt, ot) and np.array_equal(ga, oa)


def test_check_quality_matches_oracle(gpu, oracle_mod):
    pts = fx.uniform(5000, 21)
    r = gpu.delaunay(pts)
    v, interior = gpu.check_quality(pts, r)
    assert v == 0 == oracle_mod.check_delaunay_quality(pts, r.tets, r.adjacency)
    assert interior == int((r.tets < len(pts)).all(axis=1).sum())
    # a planted mistake (two tets' vertex swapped) is caught by both
    bad = r.tets.copy()
    inner = np.nonzero((bad < len(pts)).all(axis=1))[0]
    t0 = int(inner[0])
    nb = int(r.adjacency[t0, 0]) >> 5
    bad[t0, 0], bad[nb, 0] = bad[nb, 0], bad[t0, 0]
    bad_res = gpu.DelaunayResult(bad, r.adjacency, r.failed_verts)
    assert gpu.check_quality(pts, bad_res)[0] == oracle_mod.check_delaunay_quality(pts, bad, r.adjacency)


def test_device_api_zero_copy(gpu, oracle_mod):
    import torch

    pts = fx.uniform(10000, 31)
    t, a = gpu.delaunay_device(torch.from_numpy(pts).cuda())
    tets = t.cpu().numpy().view(np.uint32)
    adj = a.cpu().numpy().view(np.uint32)
    r = gpu.delaunay(pts)
    c1 = oracle_mod.canonical(tets, adj, len(pts))
    c2 = oracle_mod.canonical(r.tets, r.adjacency, len(pts))
    assert np.array_equal(c1[0], c2[0]) and np.array_equal(c1[1], c2[1])


@pytest.mark.parametrize("name,make", [
    ("lattice128", lambda: fx.lattice(128)),
    ("unit_sphere1M", lambda: fx.unit_sphere(1_000_000, 2)),
    ("mixture8M", lambda: fx.mixture(8_000_000, 3)),
])
def test_full_size_properties(gpu, oracle_mod, name, make):
    """At the benchmark sizes: every point is a vertex, links are symmetric and
    share their faces, the finite tets form a 3-ball (Euler 1), and the device
    exact check finds no locally non-Delaunay interior face."""
    pts = make()
    n = len(pts)
    r = gpu.delaunay(pts)
    assert len(r.failed_verts) == 0
    fin = finite(r.tets, n)
    assert np.unique(fin).size == n + 4
    check_adjacency(r.tets, r.adjacency)
    v, interior = gpu.check_quality(pts, r)
    assert v == 0 and interior > 2 * n
    if n <= 2_100_000:
        assert euler(fin) == 1


def test_full_size_batched(gpu):
    """The batched configuration at its benchmark size (4,096 clouds of
    log-uniform sizes in [64, 65536], about 40M points): every cloud's output
    is structurally valid and passes the device exact local-Delaunay check,
    and a sample of clouds is identical to triangulating them one by one."""
    from wtet_b200.autotune import tet_set_digest

    clouds = fx.batched_clouds(4096, 4)
    res = gpu.delaunay_batched(clouds)
    assert len(res) == len(clouds)
    for pts, r in zip(clouds, res):
        n = len(pts)
        assert (r.tets == n + 4).any(axis=1).sum() == 4
        v, interior = gpu.check_quality(pts, r)
        assert v == 0 and interior > 0
    rng = np.random.default_rng(7)
    for i in rng.choice(len(clouds), 48, replace=False):
        r = res[i]
        check_adjacency(r.tets, r.adjacency)
        single = gpu.delaunay(clouds[i])
        assert tet_set_digest(single.tets) == tet_set_digest(r.tets), i


@pytest.mark.parametrize("name,make", [
    ("uniform100k", lambda: fx.uniform(100_000, 1)),
    ("lattice24", lambda: fx.lattice(24)),
])
def test_capacity_growth_matches_oracle(gpu, oracle_mod, name, make):
    """Starting at one tet slot per point forces the in-place growth of the
    tet arrays (recaptured round graph, displaced winners retried) several
    times; the output is still the oracle's."""
    r = assert_parity(gpu, oracle_mod, make(), gpu.Config(initial_capacity=8))
    assert r.stats["capacity_grows"] >= 2, r.stats


def test_capacity_growth_batched(gpu, oracle_mod):
    clouds = fx.batched_clouds(16, 11, lo=64, hi=20000)
    res = gpu.delaunay_batched(clouds, gpu.Config(initial_capacity=8))
    assert res[0].stats["capacity_grows"] >= 2
    for pts, r in zip(clouds, res):
        tets, adj, _ = oracle_mod.delaunay(pts, 1)
        gt, ga = oracle_mod.canonical(r.tets, r.adjacency, len(pts))
        ot, oa = oracle_mod.canonical(tets, adj, len(pts))
        assert np.array_equal(gt, ot) and np.array_equal(ga, oa)
