"""Seeded synthetic point clouds (numpy PCG64, float32) with the shapes of the
benchmark configurations and of the reference's test generators
(src/tests.rs:1094-1192): uniform cube, exact lattice, unit sphere, thin
shell, Gaussian clusters, the 60/30/10 uniform / Gaussian-ball / shell
mixture, and batches of log-uniform-sized clouds."""
from __future__ import annotations

import numpy as np


def uniform(n, seed):
    return np.random.default_rng(seed).random((n, 3), dtype=np.float32)


def lattice(k):
    """k^3 points float32(i)/float32(k-1), x slowest (exact grid: SoS stress)."""
    c = (np.arange(k, dtype=np.float32) / np.float32(k - 1)).astype(np.float32)
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1).astype(np.float32)


def unit_sphere(n, seed):
    g = np.random.default_rng(seed).standard_normal((n, 3))
    return (g / np.linalg.norm(g, axis=1, keepdims=True)).astype(np.float32)


def sphere_shell(n, seed, radius=0.4, thickness=1e-4):
    """Thin shell around (0.5,0.5,0.5) (src/tests.rs:1121-1149 shape)."""
    r = np.random.default_rng(seed)
    d = r.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rad = radius + (r.random(n) - 0.5) * thickness
    return (0.5 + rad[:, None] * d).astype(np.float32)


def clustered(n, k, seed, sigma=0.05):
    """Gaussian clusters clipped to [0,1] (src/tests.rs:1152-1192 shape)."""
    r = np.random.default_rng(seed)
    centers = r.random((k, 3)) * 0.8 + 0.1
    ci = r.integers(0, k, n)
    p = centers[ci] + sigma * r.standard_normal((n, 3))
    return np.clip(p, 0.0, 1.0).astype(np.float32)


def mixture(n, seed):
    """60% uniform, 30% Gaussian ball (0.5, sigma 0.1), 10% shell r=0.4 +-1e-4, shuffled."""
    r = np.random.default_rng(seed)
    nu = int(round(0.6 * n))
    ng = int(round(0.3 * n))
    ns = n - nu - ng
    u = r.random((nu, 3))
    g = 0.5 + 0.1 * r.standard_normal((ng, 3))
    d = r.standard_normal((ns, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    s = 0.5 + (0.4 + 1e-4 * r.standard_normal(ns))[:, None] * d
    p = np.concatenate([u, g, s]).astype(np.float32)
    return p[r.permutation(n)]


def batched_sizes(num, seed, lo=64, hi=65536):
    r = np.random.default_rng(seed)
    return np.floor(np.exp(r.uniform(np.log(lo), np.log(hi), num))).astype(np.int64)


def batched_clouds(num, seed, lo=64, hi=65536):
    """Clouds of log-uniform sizes, each uniform / Gaussian / shell / jittered lattice."""
    r = np.random.default_rng(seed)
    sizes = np.floor(np.exp(r.uniform(np.log(lo), np.log(hi), num))).astype(np.int64)
    kinds = r.integers(0, 4, num)
    clouds = []
    for n, k in zip(sizes, kinds):
        n = int(n)
        if k == 0:
            p = r.random((n, 3))
        elif k == 1:
            p = 0.5 + 0.1 * r.standard_normal((n, 3))
        elif k == 2:
            d = r.standard_normal((n, 3))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            p = 0.5 + (0.4 + 1e-4 * r.standard_normal(n))[:, None] * d
        else:
            m = int(np.ceil(n ** (1.0 / 3.0)))
            g = np.stack(np.meshgrid(*[np.arange(m)] * 3, indexing="ij"), -1).reshape(-1, 3)[:n] / m
            p = g + 1e-6 * r.uniform(-1, 1, (n, 3))
        clouds.append(p.astype(np.float32))
    return clouds
