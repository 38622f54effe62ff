"""Structural validators ported from src/tests.rs:425-1090 (adjacency
consistency, Euler characteristic, orientation) in numpy.  The exact
local-Delaunay checks live in the oracle (C++)."""
import numpy as np

INVALID = 0xFFFFFFFF


def check_adjacency(tets, adj):
    """Every link is symmetric and the two tets share the three face vertices
    (src/tests.rs:425-540)."""
    tets = np.asarray(tets, np.int64)
    adj = np.asarray(adj, np.uint32)
    m = tets.shape[0]
    t_idx = np.repeat(np.arange(m), 4)
    f_idx = np.tile(np.arange(4), m)
    a = adj.reshape(-1)
    ok = a != INVALID
    t_idx, f_idx, a = t_idx[ok], f_idx[ok], a[ok].astype(np.int64)
    nb = a >> 5
    nf = a & 3
    assert (nb < m).all(), "neighbour out of range"
    back = adj[nb, nf].astype(np.int64)
    assert (back == ((t_idx << 5) | f_idx)).all(), "adjacency is not symmetric"
    # face vertices agree: sorted vertices of tet minus slot f == neighbour minus slot nf
    def face(tt, ff):
        rows = tets[tt]
        mask = np.ones_like(rows, bool)
        mask[np.arange(rows.shape[0]), ff] = False
        return np.sort(rows[mask].reshape(-1, 3), axis=1)
    assert np.array_equal(face(t_idx, f_idx), face(nb, nf)), "linked tets do not share the face"
    return True


def euler(tets):
    """V - E + F - T over the given tets (src/tests.rs:902-946); 1 for a 3-ball."""
    tets = np.sort(np.asarray(tets, np.int64), axis=1)
    V = np.unique(tets).size
    pairs = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    E = np.unique(np.concatenate([tets[:, i] * (1 << 32) + tets[:, j] for i, j in pairs])).size
    tri = [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]
    base = int(tets.max()) + 1
    Fc = np.unique(np.concatenate([(tets[:, i] * base + tets[:, j]) * base + tets[:, k] for i, j, k in tri])).size
    return V - E + Fc - tets.shape[0]


def finite(tets, n):
    tets = np.asarray(tets)
    return tets[~(tets == n + 4).any(axis=1)]
