"""wtet_b200: B200-native (sm_100a) exact 3D Delaunay tetrahedralization.

Drop-in for half-potato/wtet's Python package (python/wtet/__init__.py:48-69):

    >>> import numpy as np, wtet_b200 as wtet
    >>> pts = np.random.rand(1000, 3).astype(np.float32)
    >>> res = wtet.delaunay(pts)
    >>> res.tets.shape, res.adjacency.shape        # (M, 4) uint32 each
    >>> wtet.decode_adjacency(res.adjacency[0, 0])  # (tet, face)

The triangulation is computed by CUDA kernels in libwtet.so (C ABI:
include/wtet.h) with exact FP64 predicates and Simulation of Simplicity, so
the tet set is the unique SoS Delaunay triangulation of the points plus the
reference's four super vertices.  Additions over the reference:
``delaunay_batched`` (many clouds in one device pass), ``delaunay_device``
(zero-copy torch CUDA tensors) and ``Config(vote="learned")``.
"""
from ._core import (  # noqa: F401
    INVALID,
    Config,
    DelaunayResult,
    __version__,
    canonical,
    canonical_device,
    canonical_digest,
    check_quality,
    decode_adjacency,
    delaunay,
    delaunay_batched,
    delaunay_device,
    encode_adjacency,
    gpu_info,
    initialize_gpu,
    verify,
    verify_device,
)

__all__ = [
    "delaunay",
    "delaunay_batched",
    "delaunay_device",
    "Config",
    "DelaunayResult",
    "check_quality",
    "verify",
    "verify_device",
    "canonical",
    "canonical_device",
    "canonical_digest",
    "decode_adjacency",
    "encode_adjacency",
    "initialize_gpu",
    "gpu_info",
    "INVALID",
    "__version__",
]
