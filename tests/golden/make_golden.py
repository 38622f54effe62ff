"""Regenerates tests/golden/golden.npz: small seeded inputs and their
canonical triangulations (sorted tets + canonical adjacency) from the oracle.

The reference (Rust + wgpu) cannot be built or run here, so these fixtures pin
the oracle's restatement of its exact semantics between revisions and are the
expected outputs of the GPU parity tests.  Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import fixtures as fx  # noqa: E402
import oracle  # noqa: E402

CASES = {
    "four": np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32),
    "cube": fx.cube(),
    "icosahedron": fx.icosahedron(),
    "grid4": fx.lattice(4),
    "grid6": fx.lattice(6),
    "shell200": fx.sphere_shell(200, 42),
    "uniform500": fx.uniform(500, 1),
    "clusters300": fx.clustered(300, 3, 5),
    "mixture400": fx.mixture(400, 3),
    "coplanar_offset": fx.coplanar_with_offset(),
    "near_collinear": fx.near_collinear(),
    "duplicates": fx.with_duplicates(),
}


def main():
    out = {"names": np.array(sorted(CASES))}
    for name, pts in CASES.items():
        tets, adj, _ = oracle.delaunay(pts, 1)
        ct, ca = oracle.canonical(tets, adj, len(pts))
        out[f"{name}/points"] = pts
        out[f"{name}/tets"] = ct
        out[f"{name}/adjacency"] = ca
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", len(CASES), "cases")


if __name__ == "__main__":
    main()
