"""Seeded point generators for the parity tests (shapes of src/tests.rs:1094-1192
and of the benchmark configurations; numpy PCG64 seeds, float32).  The cloud
generators are the package's own (wtet_b200.synthetic); the small special
sets below come from the reference's unit tests."""
import numpy as np

from wtet_b200.synthetic import (  # noqa: F401
    batched_clouds,
    batched_sizes,
    clustered,
    lattice,
    mixture,
    sphere_shell,
    uniform,
    unit_sphere,
)


def cube():
    return np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [0, 0, 1], [1, 0, 1], [0, 1, 1], [1, 1, 1]],
                    np.float32)


def icosahedron():
    phi = np.float32((1.0 + np.sqrt(np.float32(5.0))) / 2.0)
    v = np.array([[-1, phi, 0], [1, phi, 0], [-1, -phi, 0], [1, -phi, 0], [0, -1, phi], [0, 1, phi],
                  [0, -1, -phi], [0, 1, -phi], [phi, 0, -1], [phi, 0, 1], [-phi, 0, -1], [-phi, 0, 1]],
                 np.float32)
    return (v * np.float32(0.3) + np.float32(0.5)).astype(np.float32)


def coplanar_with_offset():
    pts = [[ix * 0.33, iy * 0.33, 0.0] for ix in range(4) for iy in range(4)]
    pts += [[ix * 0.5 + 0.25, iy * 0.5 + 0.25, 1.0] for ix in range(2) for iy in range(2)]
    return np.array(pts, np.float32)


def near_collinear(seed=22222):
    r = np.random.default_rng(seed)
    return np.array([[i / 9.0, 0.5 + r.random() * 0.001, 0.5 + r.random() * 0.001] for i in range(10)],
                    np.float32)


def with_duplicates(seed=33333):
    p = uniform(20, seed)
    return np.concatenate([p, p[:5]]).astype(np.float32)
