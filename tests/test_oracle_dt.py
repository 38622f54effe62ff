"""The oracle triangulation against the reference's structural known answers
(src/tests.rs:286-422, 1372-1436, 1601-1630, 1715-1781): every face locally
Delaunay under exact SoS predicates, consistent orientation and adjacency,
Euler characteristic of a 3-ball, and independence of insertion order (the
SoS Delaunay triangulation is unique).  CPU only."""
import numpy as np
import pytest

import fixtures as fx
from validators import check_adjacency, euler

CASES = {
    "four": lambda: np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32),
    "cube": fx.cube,
    "icosahedron": fx.icosahedron,
    "grid4": lambda: fx.lattice(4),
    "grid5": lambda: fx.lattice(5),
    "shell30": lambda: fx.sphere_shell(30, 42),
    "random1000": lambda: fx.uniform(1000, 7),
    "clusters": lambda: fx.clustered(500, 2, 9),
    "coplanar_offset": fx.coplanar_with_offset,
    "near_collinear": fx.near_collinear,
    "duplicates": fx.with_duplicates,
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_structure(oracle_mod, name):
    pts = CASES[name]()
    n = len(pts)
    tets, adj, st = oracle_mod.delaunay(pts, 1)
    assert st["num_tets"] == len(tets) > 0
    check_adjacency(tets, adj)
    assert oracle_mod.check_orientation(pts, tets) == 0
    assert oracle_mod.check_local_delaunay(pts, tets, adj) == 0
    assert oracle_mod.check_delaunay_quality(pts, tets, adj) == 0
    assert euler(tets) == 1
    # every input point is a vertex, except exact duplicates (reported instead)
    failed = set(st["failed"].tolist())
    assert set(np.unique(tets).tolist()) == set(range(n + 4)) - failed
    if name == "duplicates":
        assert failed == set(range(20, 25))
    else:
        assert not failed


@pytest.mark.parametrize("name", ["cube", "grid4", "random1000", "duplicates", "icosahedron"])
def test_oracle_order_independent(oracle_mod, name):
    pts = CASES[name]()
    n = len(pts)
    a = oracle_mod.canonical(*oracle_mod.delaunay(pts, 0)[:2], n)
    b = oracle_mod.canonical(*oracle_mod.delaunay(pts, 1)[:2], n)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_oracle_matches_golden(oracle_mod):
    """The committed fixtures (tests/golden/make_golden.py) still reproduce."""
    import os

    path = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")
    g = np.load(path)
    for name in g["names"]:
        pts = g[f"{name}/points"]
        tets, adj, _ = oracle_mod.delaunay(pts, 1)
        ct, ca = oracle_mod.canonical(tets, adj, len(pts))
        assert np.array_equal(ct, g[f"{name}/tets"]), name
        assert np.array_equal(ca, g[f"{name}/adjacency"]), name


def test_canonical_detects_bad_adjacency(oracle_mod):
    """A mistake planted in the oracle's output changes the canonical form."""
    pts = fx.uniform(50, 3)
    tets, adj, _ = oracle_mod.delaunay(pts, 1)
    ct, ca = oracle_mod.canonical(tets, adj, len(pts))
    bad = adj.copy()
    i = int(np.nonzero(bad[:, 0] != 0xFFFFFFFF)[0][0])
    bad[i, 0] ^= 1 << 5
    ct2, ca2 = oracle_mod.canonical(tets, bad, len(pts))
    assert not np.array_equal(ca, ca2)
