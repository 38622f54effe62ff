"""The canonical parity form and the stored full-size oracle digests (CPU):
the oracle's C++ canonicaliser agrees with its numpy restatement, the oracle
reproduces a stored digest, the digest files cover every benchmark
configuration, and the reference's import name ``wtet`` serves the library."""
import json
import os

import numpy as np

import fixtures as fx

HERE = os.path.dirname(os.path.abspath(__file__))


def test_canonical_cpp_matches_numpy(oracle_mod):
    for pts in (fx.uniform(3000, 4), fx.lattice(7), fx.with_duplicates(), fx.cube()):
        tets, adj, _ = oracle_mod.delaunay(pts, 1)
        a = oracle_mod.canonical(tets, adj, len(pts))
        b = oracle_mod.canonical_numpy(tets, adj, len(pts))
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        # row order of the input does not matter
        perm = np.random.default_rng(1).permutation(len(tets))
        inv = np.empty_like(perm)
        inv[perm] = np.arange(len(perm))
        adj2 = adj[perm].copy()
        ok = adj2 != oracle_mod.INVALID
        adj2[ok] = (inv[adj2[ok] >> 5].astype(np.uint32) << 5) | (adj2[ok] & 3)
        c = oracle_mod.canonical(tets[perm], adj2, len(pts))
        assert np.array_equal(a[0], c[0]) and np.array_equal(a[1], c[1])


def test_stored_digest_reproduced(oracle_mod):
    with open(os.path.join(HERE, "golden", "full_size.json")) as f:
        g = json.load(f)
    pts = fx.uniform(100_000, 1)
    tets, adj, _ = oracle_mod.delaunay(pts, 1)
    assert oracle_mod.digest(*oracle_mod.canonical(tets, adj, len(pts))) == g["uniform100k"]["sha256"]


def test_digest_files_cover_the_benchmarks():
    with open(os.path.join(HERE, "golden", "full_size.json")) as f:
        g = json.load(f)
    want = {"uniform100k", "lattice128", "unit_sphere1M", "mixture8M_s3"} | {f"mixture8M_s{s}" for s in range(101, 106)}
    assert want <= set(g)
    assert g["lattice128"]["n"] == 128 ** 3 and g["mixture8M_s3"]["n"] == 8_000_000
    b = np.load(os.path.join(HERE, "golden", "batched_digests.npz"))
    assert b["digests"].shape == (4096, 32)
    assert np.array_equal(b["sizes"], np.array([len(c) for c in fx.batched_clouds(4096, 4)]))


def test_wtet_import_name(wt):
    import wtet
    import wtet._core

    assert wtet.delaunay is wt.delaunay and wtet.Config is wt.Config
    assert wtet._core.check_quality is wt.check_quality
    for name in ("delaunay", "Config", "DelaunayResult", "decode_adjacency", "encode_adjacency", "initialize_gpu",
                 "gpu_info", "INVALID", "__version__"):
        assert hasattr(wtet, name), name
    assert wtet.decode_adjacency(wtet.encode_adjacency(9, 3)) == (9, 3)


def test_package_digest_matches_oracle_digest(wt, oracle_mod):
    rng = np.random.default_rng(3)
    t = rng.integers(0, 2 ** 32, (50, 4), dtype=np.uint64).astype(np.uint32)
    a = rng.integers(0, 2 ** 32, (50, 4), dtype=np.uint64).astype(np.uint32)
    assert wt.canonical_digest(t, a) == oracle_mod.digest(t, a)
