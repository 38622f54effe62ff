"""ctypes binding of libwtet.so, mirroring the reference's ``wtet._core``
module (src/python.rs:166-402): ``delaunay``, ``Config``, ``DelaunayResult``,
``check_quality``, ``encode_adjacency`` / ``decode_adjacency``,
``initialize_gpu``, ``gpu_info``, ``INVALID`` and ``__version__`` -- same
names, argument meaning and error behaviour (ValueError for bad input, shape
or insertion rule; RuntimeError for device failures).

The triangulation runs only on the CUDA path: if libwtet.so is missing or no
GPU is present, calls raise; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libwtet.so")

INVALID = 0xFFFFFFFF
__version__ = "0.1.0"

WTET_OK = 0
WTET_ERR_ARG = -1
WTET_ERR_CAPACITY = -2


class _Config(ctypes.Structure):
    _fields_ = [
        ("insertion_rule", ctypes.c_uint32),
        ("enable_flipping", ctypes.c_uint32),
        ("enable_sorting", ctypes.c_uint32),
        ("enable_hilbert_sorting", ctypes.c_uint32),
        ("enable_splaying", ctypes.c_uint32),
        ("max_insert_iterations", ctypes.c_uint32),
        ("max_flip_iterations", ctypes.c_uint32),
        ("vote_mode", ctypes.c_uint32),
        ("block_size", ctypes.c_uint32),
        ("rounds_per_graph", ctypes.c_uint32),
        ("overlap_shift", ctypes.c_uint32),
        ("candidate_filter", ctypes.c_uint32),
        ("pool_factor", ctypes.c_uint32),
        ("learned_gate", ctypes.c_uint32),
        ("initial_capacity", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32 * 1),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("rounds", ctypes.c_uint32),
        ("strata", ctypes.c_uint32),
        ("inserted", ctypes.c_uint64),
        ("candidates", ctypes.c_uint64),
        ("big_cavities", ctypes.c_uint64),
        ("tets_created", ctypes.c_uint64),
        ("num_tets", ctypes.c_uint64),
        ("walk_steps", ctypes.c_uint64),
        ("num_failed", ctypes.c_uint64),
        ("kernel_launches", ctypes.c_uint64),
        ("device_ms", ctypes.c_double),
        ("vote_winners", ctypes.c_uint64),
        ("capacity_grows", ctypes.c_uint64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class _Result(ctypes.Structure):
    _fields_ = [
        ("tets", ctypes.POINTER(ctypes.c_uint32)),
        ("adjacency", ctypes.POINTER(ctypes.c_uint32)),
        ("failed_verts", ctypes.POINTER(ctypes.c_uint32)),
        ("num_tets", ctypes.c_uint64),
        ("num_failed", ctypes.c_uint64),
        ("stats", Stats),
    ]


_lib = None
EXPORTS = (
    "wtet_config_default",
    "wtet_delaunay",
    "wtet_delaunay_into",
    "wtet_delaunay_device",
    "wtet_delaunay_batched",
    "wtet_check_quality",
    "wtet_max_tets",
    "wtet_result_free",
    "wtet_last_error",
    "wtet_initialize_gpu",
    "wtet_gpu_info",
    "wtet_version",
    "wtet_learned_set_weights",
    "wtet_learned_has_weights",
    "wtet_learned_collect",
    "wtet_mlp_loss_grad",
    "wtet_mlp_train",
    "wtet_mlp_score",
    "wtet_autotune_set_table",
    "wtet_autotune_get_table",
    "wtet_autotune_resolve",
    "wtet_morton_index",
    "wtet_hilbert_index",
    "wtet_verify",
    "wtet_verify_device",
    "wtet_canonicalize",
    "wtet_canonicalize_device",
    "wtet_predicate_signs",
)


class VerifyReport(ctypes.Structure):
    _fields_ = [
        ("finite_tets", ctypes.c_uint64),
        ("faces_checked", ctypes.c_uint64),
        ("violations", ctypes.c_uint64),
        ("misoriented", ctypes.c_uint64),
        ("broken_links", ctypes.c_uint64),
        ("hull_faces", ctypes.c_uint64),
        ("bad_vertex_ids", ctypes.c_uint64),
    ]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class TrainConfig(ctypes.Structure):
    _fields_ = [
        ("epochs", ctypes.c_uint32),
        ("batch", ctypes.c_uint32),
        ("lr", ctypes.c_float),
        ("beta1", ctypes.c_float),
        ("beta2", ctypes.c_float),
        ("eps", ctypes.c_float),
        ("seed", ctypes.c_uint64),
    ]


def lib_path() -> str:
    return _LIB_PATH


def load():
    """Loads libwtet.so (raises ImportError if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError(
            "wtet_b200: libwtet.so is missing; build it with `python -m wtet_b200.build` "
            "(the CUDA path has no fallback)"
        )
    L = ctypes.CDLL(_LIB_PATH)
    P = ctypes.c_void_p
    u64 = ctypes.c_uint64
    L.wtet_config_default.argtypes = [ctypes.POINTER(_Config)]
    L.wtet_config_default.restype = None
    L.wtet_delaunay.argtypes = [P, u64, ctypes.POINTER(_Config), ctypes.POINTER(_Result)]
    L.wtet_delaunay.restype = ctypes.c_int
    L.wtet_delaunay_into.argtypes = [P, u64, ctypes.POINTER(_Config), P, P, u64, ctypes.POINTER(u64), P,
                                     ctypes.POINTER(Stats)]
    L.wtet_delaunay_into.restype = ctypes.c_int
    L.wtet_delaunay_device.argtypes = [P, u64, ctypes.POINTER(_Config), P, P, u64, ctypes.POINTER(u64),
                                       ctypes.POINTER(Stats), P]
    L.wtet_delaunay_device.restype = ctypes.c_int
    L.wtet_delaunay_batched.argtypes = [P, P, ctypes.c_uint32, ctypes.POINTER(_Config), P, P, u64, P,
                                        ctypes.POINTER(Stats)]
    L.wtet_delaunay_batched.restype = ctypes.c_int
    L.wtet_check_quality.argtypes = [P, u64, P, P, u64, ctypes.POINTER(u64), ctypes.POINTER(u64)]
    L.wtet_check_quality.restype = ctypes.c_int
    L.wtet_max_tets.argtypes = [u64]
    L.wtet_max_tets.restype = u64
    L.wtet_result_free.argtypes = [ctypes.POINTER(_Result)]
    L.wtet_result_free.restype = None
    L.wtet_last_error.restype = ctypes.c_char_p
    L.wtet_initialize_gpu.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    L.wtet_initialize_gpu.restype = ctypes.c_int
    L.wtet_gpu_info.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    L.wtet_gpu_info.restype = ctypes.c_int
    L.wtet_version.restype = ctypes.c_char_p
    L.wtet_learned_set_weights.argtypes = [P, u64]
    L.wtet_learned_set_weights.restype = ctypes.c_int
    L.wtet_learned_has_weights.argtypes = []
    L.wtet_learned_has_weights.restype = ctypes.c_int
    L.wtet_learned_collect.argtypes = [P, P, ctypes.c_uint32, ctypes.POINTER(_Config), ctypes.c_uint32, P, P, u64,
                                       ctypes.POINTER(u64), ctypes.POINTER(Stats)]
    L.wtet_learned_collect.restype = ctypes.c_int
    L.wtet_mlp_loss_grad.argtypes = [P, P, u64, P, P, P]
    L.wtet_mlp_loss_grad.restype = ctypes.c_int
    L.wtet_mlp_train.argtypes = [P, P, u64, ctypes.POINTER(TrainConfig), P, P]
    L.wtet_mlp_train.restype = ctypes.c_int
    L.wtet_mlp_score.argtypes = [P, u64, P]
    L.wtet_mlp_score.restype = ctypes.c_int
    L.wtet_autotune_set_table.argtypes = [P, ctypes.c_uint32]
    L.wtet_autotune_set_table.restype = ctypes.c_int
    L.wtet_autotune_get_table.argtypes = [P, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]
    L.wtet_autotune_get_table.restype = ctypes.c_int
    L.wtet_autotune_resolve.argtypes = [ctypes.POINTER(_Config), u64, ctypes.c_uint32, ctypes.POINTER(_Config)]
    L.wtet_autotune_resolve.restype = ctypes.c_int
    L.wtet_morton_index.argtypes = [ctypes.c_uint32] * 3
    L.wtet_morton_index.restype = ctypes.c_uint32
    L.wtet_hilbert_index.argtypes = [ctypes.c_uint32] * 4
    L.wtet_hilbert_index.restype = ctypes.c_uint32
    L.wtet_verify.argtypes = [P, u64, P, P, u64, ctypes.POINTER(VerifyReport)]
    L.wtet_verify.restype = ctypes.c_int
    L.wtet_verify_device.argtypes = [P, u64, P, P, u64, ctypes.POINTER(VerifyReport), P]
    L.wtet_verify_device.restype = ctypes.c_int
    L.wtet_canonicalize.argtypes = [P, P, u64, u64, P, P, ctypes.POINTER(u64)]
    L.wtet_canonicalize.restype = ctypes.c_int
    L.wtet_canonicalize_device.argtypes = [P, P, u64, u64, P, P, ctypes.POINTER(u64), P]
    L.wtet_canonicalize_device.restype = ctypes.c_int
    L.wtet_predicate_signs.argtypes = [P, P, u64, P, P]
    L.wtet_predicate_signs.restype = ctypes.c_int
    _lib = L
    _install_packaged_table()
    return L


def _install_packaged_table():
    """Installs the autotuner table shipped with the package, if present."""
    if os.path.exists(os.path.join(_HERE, "data", "autotune.json")):
        from . import autotune

        autotune.load()


def _raise(status: int):
    msg = load().wtet_last_error().decode(errors="replace")
    if status == WTET_ERR_ARG:
        raise ValueError(msg)
    raise RuntimeError(f"wtet_b200 error {status}: {msg}")


_RULES = {"circumcenter": 0, "centroid": 1}
_VOTES = {"plain": 0, "learned": 1}


class Config:
    """Configuration, as ``wtet.Config`` (src/python.rs:53-117, src/types.rs:32-61).

    ``vote`` ("plain" or "learned") selects the insertion scheduler;
    ``block_size``, ``rounds_per_graph``, ``overlap_shift``,
    ``candidate_filter`` and ``pool_factor`` are performance knobs (0 = the
    autotuner's value for the job's size, see wtet_b200.autotune);
    ``learned_gate`` bounds the rounds the learned scheduler serves (rounds
    that may see at most learned_gate x 1024 uninserted points; 0 = 2048);
    ``initial_capacity`` sets the initial tet slots per point in eighths (0 =
    9 per point; smaller values exercise the in-place growth of the tet
    arrays).  No option changes the resulting triangulation."""

    def __init__(self, insertion_rule: str = "circumcenter", enable_flipping: bool = True,
                 enable_sorting: bool = False, enable_hilbert_sorting: bool = False,
                 enable_splaying: bool = True, max_insert_iterations: int = 100,
                 max_flip_iterations: int = 10, vote: str = "plain", block_size: int = 0,
                 rounds_per_graph: int = 0, overlap_shift: int = 0, candidate_filter: int = 0,
                 pool_factor: int = 0, learned_gate: int = 0, initial_capacity: int = 0):
        rule = str(insertion_rule).lower()
        if rule not in _RULES:
            raise ValueError(
                f"Invalid insertion_rule '{insertion_rule}'. Must be 'circumcenter' or 'centroid'."
            )
        if vote not in _VOTES:
            raise ValueError(f"Invalid vote '{vote}'. Must be 'plain' or 'learned'.")
        self.insertion_rule = rule
        self.enable_flipping = bool(enable_flipping)
        self.enable_sorting = bool(enable_sorting)
        self.enable_hilbert_sorting = bool(enable_hilbert_sorting)
        self.enable_splaying = bool(enable_splaying)
        self.max_insert_iterations = int(max_insert_iterations)
        self.max_flip_iterations = int(max_flip_iterations)
        self.vote = vote
        self.block_size = int(block_size)
        self.rounds_per_graph = int(rounds_per_graph)
        self.overlap_shift = int(overlap_shift)
        self.candidate_filter = int(candidate_filter)
        self.pool_factor = int(pool_factor)
        self.learned_gate = int(learned_gate)
        self.initial_capacity = int(initial_capacity)

    def _c(self) -> _Config:
        if self.vote == "learned":
            _ensure_learned_weights()
        c = _Config()
        c.insertion_rule = _RULES[self.insertion_rule]
        c.enable_flipping = int(self.enable_flipping)
        c.enable_sorting = int(self.enable_sorting)
        c.enable_hilbert_sorting = int(self.enable_hilbert_sorting)
        c.enable_splaying = int(self.enable_splaying)
        c.max_insert_iterations = self.max_insert_iterations
        c.max_flip_iterations = self.max_flip_iterations
        c.vote_mode = _VOTES[self.vote]
        c.block_size = self.block_size
        c.rounds_per_graph = self.rounds_per_graph
        c.overlap_shift = self.overlap_shift
        c.candidate_filter = self.candidate_filter
        c.pool_factor = self.pool_factor
        c.learned_gate = self.learned_gate
        c.initial_capacity = self.initial_capacity
        return c

    def __repr__(self) -> str:
        return (
            f"Config(insertion_rule='{self.insertion_rule}', flipping={self.enable_flipping}, "
            f"sorting={self.enable_sorting}, hilbert={self.enable_hilbert_sorting}, "
            f"splaying={self.enable_splaying}, max_insert_iter={self.max_insert_iterations}, "
            f"max_flip_iter={self.max_flip_iterations}, vote='{self.vote}')"
        )


def _ensure_learned_weights():
    """Installs the packaged learned-vote weights unless weights are set."""
    if not load().wtet_learned_has_weights():
        from . import learned

        learned.load_default()


class DelaunayResult:
    """Result, as ``wtet.DelaunayResult`` (src/python.rs:126-160)."""

    def __init__(self, tets: np.ndarray, adjacency: np.ndarray, failed_verts: np.ndarray, stats=None):
        self.tets = tets
        self.adjacency = adjacency
        self.failed_verts = failed_verts
        self.stats = stats or {}

    @property
    def num_tets(self) -> int:
        return int(self.tets.shape[0])

    @property
    def num_failed(self) -> int:
        return int(self.failed_verts.shape[0])

    def __repr__(self) -> str:
        return f"DelaunayResult(num_tets={self.num_tets}, failed_verts={self.num_failed})"


def _points(points) -> np.ndarray:
    a = np.asarray(points)
    if a.ndim != 2 or a.shape[1] != 3:
        raise ValueError(f"Points must have shape (N, 3), got {list(a.shape)}")
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def delaunay(points, config: Config | None = None) -> DelaunayResult:
    """3D Delaunay triangulation (src/python.rs:166-257, src/lib.rs:160-310)."""
    pts = _points(points)
    n = pts.shape[0]
    if n < 4:
        raise ValueError(f"Need at least 4 points for 3D Delaunay, got {n}")
    L = load()
    cfg = (config or Config())._c()
    cap = int(L.wtet_max_tets(n))
    tets = np.empty((cap, 4), np.uint32)
    adj = np.empty((cap, 4), np.uint32)
    m = ctypes.c_uint64(0)
    st = Stats()
    failed = np.empty(n, np.uint32)
    rc = L.wtet_delaunay_into(_ptr(pts), n, ctypes.byref(cfg), _ptr(tets), _ptr(adj), cap, ctypes.byref(m),
                              _ptr(failed), ctypes.byref(st))
    if rc == WTET_ERR_CAPACITY and m.value > cap:
        cap = m.value
        tets = np.empty((cap, 4), np.uint32)
        adj = np.empty((cap, 4), np.uint32)
        rc = L.wtet_delaunay_into(_ptr(pts), n, ctypes.byref(cfg), _ptr(tets), _ptr(adj), cap,
                                  ctypes.byref(m), _ptr(failed), ctypes.byref(st))
    if rc != WTET_OK:
        _raise(rc)
    k = m.value
    # The buffers were sized for the worst case (8n + 64 rows, about 20% above
    # a typical 6.7n): shrink them in place (realloc of the tail, no second
    # multi-GB copy) so that the result holds only its own rows.
    tets.resize((k, 4), refcheck=False)
    adj.resize((k, 4), refcheck=False)
    return DelaunayResult(tets, adj, failed[: st.num_failed].copy(), st.as_dict())


def delaunay_batched(clouds, config: Config | None = None):
    """Triangulates many clouds in one device pass (no reference counterpart).

    ``clouds`` is a list of (N_i, 3) arrays, or a tuple ``(points, offsets)``
    with offsets of length num_clouds + 1.  Returns a list of DelaunayResult,
    each identical to ``delaunay`` on that cloud alone (cloud-local ids)."""
    if isinstance(clouds, tuple) and len(clouds) == 2 and np.asarray(clouds[1]).ndim == 1:
        pts = _points(clouds[0])
        offsets = np.ascontiguousarray(clouds[1], dtype=np.uint64)
    else:
        arrs = [_points(c) for c in clouds]
        if not arrs:
            return []
        offsets = np.zeros(len(arrs) + 1, np.uint64)
        offsets[1:] = np.cumsum([a.shape[0] for a in arrs])
        pts = np.ascontiguousarray(np.concatenate(arrs, axis=0))
    nc = offsets.shape[0] - 1
    sizes = np.diff(offsets.astype(np.int64))
    if nc < 1 or (sizes < 4).any():
        raise ValueError("Need at least 4 points for 3D Delaunay in every cloud")
    L = load()
    cfg = (config or Config())._c()
    cap = int(sum(int(L.wtet_max_tets(int(s))) for s in sizes))
    tets = np.empty((cap, 4), np.uint32)
    adj = np.empty((cap, 4), np.uint32)
    toff = np.zeros(nc + 1, np.uint64)
    st = Stats()
    rc = L.wtet_delaunay_batched(_ptr(pts), _ptr(offsets), nc, ctypes.byref(cfg), _ptr(tets), _ptr(adj), cap,
                                 _ptr(toff), ctypes.byref(st))
    if rc == WTET_ERR_CAPACITY and int(toff[-1]) > cap:
        cap = int(toff[-1])
        tets = np.empty((cap, 4), np.uint32)
        adj = np.empty((cap, 4), np.uint32)
        rc = L.wtet_delaunay_batched(_ptr(pts), _ptr(offsets), nc, ctypes.byref(cfg), _ptr(tets), _ptr(adj),
                                     cap, _ptr(toff), ctypes.byref(st))
    if rc != WTET_OK:
        _raise(rc)
    out = []
    stats = st.as_dict()
    for c in range(nc):
        a, b = int(toff[c]), int(toff[c + 1])
        out.append(DelaunayResult(tets[a:b], adj[a:b], np.zeros(0, np.uint32), stats))
    return out


def delaunay_device(points, config: Config | None = None, with_stats: bool = False):
    """Zero-copy variant for a CUDA torch tensor of shape (N, 3), float32.

    Returns (tets, adjacency) as CUDA int32-viewed uint32 tensors of shape
    (M, 4), computed on torch's current stream; with ``with_stats`` also the
    call's statistics (the ``stats`` dict of DelaunayResult)."""
    import torch

    if not (isinstance(points, torch.Tensor) and points.is_cuda):
        raise ValueError("delaunay_device expects a CUDA torch tensor")
    if points.dim() != 2 or points.shape[1] != 3:
        raise ValueError(f"Points must have shape (N, 3), got {list(points.shape)}")
    pts = points.contiguous().to(torch.float32)
    n = pts.shape[0]
    if n < 4:
        raise ValueError(f"Need at least 4 points for 3D Delaunay, got {n}")
    L = load()
    cfg = (config or Config())._c()
    cap = int(L.wtet_max_tets(n))
    stream = ctypes.c_void_p(torch.cuda.current_stream(pts.device).cuda_stream)
    m = ctypes.c_uint64(0)
    st = Stats()
    for _ in range(2):
        tets = torch.empty((cap, 4), dtype=torch.int32, device=pts.device)
        adj = torch.empty((cap, 4), dtype=torch.int32, device=pts.device)
        rc = L.wtet_delaunay_device(ctypes.c_void_p(pts.data_ptr()), n, ctypes.byref(cfg),
                                    ctypes.c_void_p(tets.data_ptr()), ctypes.c_void_p(adj.data_ptr()), cap,
                                    ctypes.byref(m), ctypes.byref(st), stream)
        if rc == WTET_ERR_CAPACITY and m.value > cap:
            cap = m.value
            continue
        break
    if rc != WTET_OK:
        _raise(rc)
    if with_stats:
        return tets[: m.value], adj[: m.value], st.as_dict()
    return tets[: m.value], adj[: m.value]


def check_quality(points, result: DelaunayResult):
    """(violations, interior_tets), as ``wtet._core.check_quality``
    (src/python.rs:282-341, src/lib.rs:25-78), evaluated on the device."""
    pts = _points(points)
    n = pts.shape[0]
    t = np.ascontiguousarray(result.tets, np.uint32).reshape(-1, 4)
    a = np.ascontiguousarray(result.adjacency, np.uint32).reshape(-1, 4)
    v = ctypes.c_uint64(0)
    i = ctypes.c_uint64(0)
    L = load()
    rc = L.wtet_check_quality(_ptr(pts), n, _ptr(t), _ptr(a), t.shape[0], ctypes.byref(v), ctypes.byref(i))
    if rc != WTET_OK:
        _raise(rc)
    return int(v.value), int(i.value)


def verify(points, result: DelaunayResult) -> dict:
    """Every-face exact verification on the device (extends check_quality,
    src/lib.rs:25-78, to faces with super vertices; checks orientation and
    links too).  A complete output has violations = misoriented =
    broken_links = bad_vertex_ids = 0 and hull_faces = 4."""
    pts = _points(points)
    t = np.ascontiguousarray(result.tets, np.uint32).reshape(-1, 4)
    a = np.ascontiguousarray(result.adjacency, np.uint32).reshape(-1, 4)
    rep = VerifyReport()
    rc = load().wtet_verify(_ptr(pts), pts.shape[0], _ptr(t), _ptr(a), t.shape[0], ctypes.byref(rep))
    if rc != WTET_OK:
        _raise(rc)
    return rep.as_dict()


def verify_device(points, tets, adjacency) -> dict:
    """verify() on CUDA torch tensors (points (N,3) f32; tets, adjacency
    (M,4) 32-bit), on torch's current stream."""
    import torch

    rep = VerifyReport()
    stream = ctypes.c_void_p(torch.cuda.current_stream(points.device).cuda_stream)
    rc = load().wtet_verify_device(ctypes.c_void_p(points.data_ptr()), points.shape[0],
                                   ctypes.c_void_p(tets.data_ptr()), ctypes.c_void_p(adjacency.data_ptr()),
                                   tets.shape[0], ctypes.byref(rep), stream)
    if rc != WTET_OK:
        _raise(rc)
    return rep.as_dict()


def canonical(tets, adjacency, n: int):
    """Canonical parity form, computed on the device: tets without the
    infinity vertex n+4, ids sorted per row, rows sorted; adjacency re-indexed
    to that order ((neighbour << 5) | sorted slot of its opposite vertex,
    INVALID towards a missing or infinity neighbour).  Returns numpy
    (K,4) uint32 arrays."""
    t = np.ascontiguousarray(tets, np.uint32).reshape(-1, 4)
    a = np.ascontiguousarray(adjacency, np.uint32).reshape(-1, 4)
    m = t.shape[0]
    ot = np.empty((max(m, 1), 4), np.uint32)
    oa = np.empty((max(m, 1), 4), np.uint32)
    k = ctypes.c_uint64(0)
    rc = load().wtet_canonicalize(_ptr(t), _ptr(a), m, int(n), _ptr(ot), _ptr(oa), ctypes.byref(k))
    if rc != WTET_OK:
        _raise(rc)
    ot.resize((k.value, 4), refcheck=False)
    oa.resize((k.value, 4), refcheck=False)
    return ot, oa


def canonical_device(tets, adjacency, n: int):
    """canonical() on CUDA torch tensors; returns CUDA tensors (K,4)."""
    import torch

    m = tets.shape[0]
    ot = torch.empty((max(m, 1), 4), dtype=torch.int32, device=tets.device)
    oa = torch.empty((max(m, 1), 4), dtype=torch.int32, device=tets.device)
    k = ctypes.c_uint64(0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(tets.device).cuda_stream)
    rc = load().wtet_canonicalize_device(ctypes.c_void_p(tets.data_ptr()), ctypes.c_void_p(adjacency.data_ptr()), m,
                                         int(n), ctypes.c_void_p(ot.data_ptr()), ctypes.c_void_p(oa.data_ptr()),
                                         ctypes.byref(k), stream)
    if rc != WTET_OK:
        _raise(rc)
    return ot[: k.value], oa[: k.value]


def canonical_digest(canon_tets, canon_adjacency) -> str:
    """SHA-256 of a canonical form: the tets' bytes, then the adjacency's
    (little-endian u32)."""
    import hashlib

    h = hashlib.sha256()
    for arr in (canon_tets, canon_adjacency):
        if hasattr(arr, "cpu"):
            arr = arr.cpu().numpy()
        h.update(np.ascontiguousarray(arr).view(np.uint32).astype("<u4", copy=False).tobytes())
    return h.hexdigest()


def predicate_signs(points5, keys5):
    """(orient3d_sos of the first four points, orient4d of all five) per
    record, as the device's insertion rounds evaluate them: points5 (m, 5, 3)
    float32 used as given, keys5 (m, 5) uint32 SoS keys."""
    p = np.ascontiguousarray(points5, np.float32).reshape(-1, 15)
    k = np.ascontiguousarray(keys5, np.uint32).reshape(-1, 5)
    m = p.shape[0]
    o3 = np.empty(m, np.int32)
    o4 = np.empty(m, np.int32)
    rc = load().wtet_predicate_signs(_ptr(p), _ptr(k), m, _ptr(o3), _ptr(o4))
    if rc != WTET_OK:
        _raise(rc)
    return o3, o4


def decode_adjacency(packed: int):
    """(tet_idx, face_idx) from (tet_idx << 5) | face_idx (src/python.rs:259-265)."""
    return (int(packed) >> 5, int(packed) & 3)


def encode_adjacency(tet_idx: int, face_idx: int) -> int:
    """(tet_idx << 5) | face_idx (src/python.rs:267-272)."""
    return ((int(tet_idx) << 5) | (int(face_idx) & 3)) & 0xFFFFFFFF


def initialize_gpu() -> str:
    buf = ctypes.create_string_buffer(1024)
    rc = load().wtet_initialize_gpu(buf, 1024)
    if rc != WTET_OK:
        _raise(rc)
    return buf.value.decode()


def gpu_info() -> str:
    buf = ctypes.create_string_buffer(1024)
    load().wtet_gpu_info(buf, 1024)
    return buf.value.decode() or "GPU not yet initialized. Call initialize_gpu() or run delaunay() to initialize."
