"""Generates tests/golden/full_size.json and tests/golden/batched_digests.npz:
the oracle's canonical tet set and adjacency, as SHA-256 digests, for every
benchmark configuration at its full size.

    python tests/golden/make_full_size.py [--jobs 4] [--only name,...]

Configurations (seeded numpy PCG64 generators of wtet_b200.synthetic):
  uniform100k      100,000 uniform points, seed 1
  lattice128       the exact 128^3 lattice float32(i)/127 (2,097,152 points)
  unit_sphere1M    1,000,000 points on the unit sphere, seed 2
  mixture8M_s3     8,000,000 points of the 60/30/10 mixture, seed 3
  mixture8M_s101..105  the same distribution, seeds 101-105
  batched          4,096 clouds of log-uniform sizes in [64, 65536], seed 4:
                   one digest per cloud (batched_digests.npz)

Each digest is oracle.digest(oracle.canonical(...)) of the oracle's
sequential exact Bowyer-Watson triangulation (the reference's
src/phase2.rs:383-606 semantics).  The GPU tests compare the library's
canonical output with these digests byte for byte (through SHA-256).
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CONFIGS = {
    "uniform100k": ("uniform", (100_000, 1)),
    "lattice128": ("lattice", (128,)),
    "unit_sphere1M": ("unit_sphere", (1_000_000, 2)),
    "mixture8M_s3": ("mixture", (8_000_000, 3)),
    **{f"mixture8M_s{s}": ("mixture", (8_000_000, s)) for s in range(101, 106)},
}


def points_for(name):
    from wtet_b200 import synthetic as syn

    fn, args = CONFIGS[name]
    return getattr(syn, fn)(*args)


def one_config(name):
    import oracle

    pts = points_for(name)
    t0 = time.perf_counter()
    tets, adj, st = oracle.delaunay(pts, 1)
    dt = time.perf_counter() - t0
    ct, ca = oracle.canonical(tets, adj, len(pts))
    return name, {"n": len(pts), "num_tets": int(tets.shape[0]), "canonical_rows": int(ct.shape[0]),
                  "failed": int(len(st["failed"])), "sha256": oracle.digest(ct, ca), "oracle_s": round(dt, 1)}


def one_cloud(args):
    import oracle

    i, pts = args
    tets, adj, st = oracle.delaunay(pts, 1)
    ct, ca = oracle.canonical(tets, adj, len(pts))
    return i, bytes.fromhex(oracle.digest(ct, ca))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=4)
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    import oracle

    oracle.build()
    only = [s for s in args.only.split(",") if s]
    names = [n for n in CONFIGS if not only or n in only]
    out_path = os.path.join(HERE, "full_size.json")
    table = {}
    if os.path.exists(out_path):
        with open(out_path) as f:
            table = json.load(f)
    ctx = mp.get_context("spawn")
    with ctx.Pool(args.jobs) as pool:
        if names:
            for name, rec in pool.imap_unordered(one_config, names):
                table[name] = rec
                print(name, rec, flush=True)
                with open(out_path, "w") as f:
                    json.dump(dict(sorted(table.items())), f, indent=1)
        if not only or "batched" in only:
            from wtet_b200 import synthetic as syn

            clouds = syn.batched_clouds(4096, 4)
            dig = np.zeros((len(clouds), 32), np.uint8)
            for i, d in pool.imap_unordered(one_cloud, list(enumerate(clouds)), chunksize=16):
                dig[i] = np.frombuffer(d, np.uint8)
            sizes = np.array([len(c) for c in clouds], np.int64)
            np.savez_compressed(os.path.join(HERE, "batched_digests.npz"), digests=dig, sizes=sizes)
            print("batched", len(clouds), int(sizes.sum()), flush=True)


if __name__ == "__main__":
    main()
