"""Point-order curves (host functions of the C ABI, no GPU needed): the
Morton index matches the reference's bit interleave (src/morton.rs:88-151,
restated by the oracle); the Hilbert index is a bijection onto the cells whose
consecutive indices are face-adjacent -- the uniqueness and locality the
reference's own Hilbert tests check (src/hilbert.rs:46-120).  On the GPU the
Hilbert order gives the same tet set as the Morton order."""
import numpy as np
import pytest

import fixtures as fx


def test_morton_matches_reference_interleave(wt, oracle_mod):
    L = wt._core.load()
    r = np.random.default_rng(3)
    for x, y, z in r.integers(0, 1024, (200, 3)):
        assert L.wtet_morton_index(int(x), int(y), int(z)) == oracle_mod.interleave_bits(int(x), int(y), int(z))


@pytest.mark.parametrize("bits", [1, 2, 3, 4, 5])
def test_hilbert_is_a_face_adjacent_bijection(wt, bits):
    L = wt._core.load()
    n = 1 << bits
    cells = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)
    idx = np.array([L.wtet_hilbert_index(int(x), int(y), int(z), bits) for x, y, z in cells])
    assert np.array_equal(np.sort(idx), np.arange(n ** 3))          # uniqueness
    order = cells[np.argsort(idx)]
    step = np.abs(np.diff(order, axis=0)).sum(axis=1)
    assert (step == 1).all()                                          # locality
    assert tuple(order[0]) == (0, 0, 0)


def test_hilbert_rejects_bad_bits(wt):
    L = wt._core.load()
    assert L.wtet_hilbert_index(1, 2, 3, 0) == 0xFFFFFFFF
    assert L.wtet_hilbert_index(1, 2, 3, 11) == 0xFFFFFFFF
    assert L.wtet_hilbert_index(1023, 1023, 1023, 10) < 1 << 30


@pytest.mark.gpu
def test_hilbert_order_gives_the_same_tets(gpu, oracle_mod):
    for pts in (fx.mixture(100_000, 8), fx.lattice(20)):
        a = gpu.delaunay(pts, gpu.Config())
        b = gpu.delaunay(pts, gpu.Config(enable_hilbert_sorting=True))
        ca = oracle_mod.canonical(a.tets, a.adjacency, len(pts))
        cb = oracle_mod.canonical(b.tets, b.adjacency, len(pts))
        assert np.array_equal(ca[0], cb[0]) and np.array_equal(ca[1], cb[1])
