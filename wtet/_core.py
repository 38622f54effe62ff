"""``wtet._core`` (src/python.rs:377-402): the module-level functions of the
reference's compiled extension, served by wtet_b200's C-ABI binding."""
from wtet_b200._core import (  # noqa: F401
    INVALID,
    Config,
    DelaunayResult,
    __version__,
    check_quality,
    decode_adjacency,
    delaunay,
    encode_adjacency,
    gpu_info,
    initialize_gpu,
)
