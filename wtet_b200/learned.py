"""Learned insertion scheduler: data collection, training and weights.

Every tet votes for its uninserted point deepest inside its circumsphere (the
reference's vote, src/shaders/vote.wgsl:401-494).  The vote winners then
compete for their cavities by claim keys: the smaller key wins a contested
tet.  The plain method hashes the keys, so in a crowded neighbourhood the
winners lose to each other round after round, and those neighbourhoods set
the number of rounds.  ``Config(vote="learned")`` lets a small MLP (12 -> 64
-> 64 -> 64 -> 1, ReLU) predict each winner's probability of inserting in
this round under hashed keys; the winners least likely to insert -- the
crowded ones -- get the smallest keys and claim first.  The network serves
the rounds of the first strata (up to ``Config.learned_gate`` x 1024
uninserted points), whose cost is a fixed overhead per round; the bulk
rounds keep hashed keys.  Inference is fused into the kernel that turns
votes into winners (BF16 tensor-core mma, FP32 accumulate); the
triangulation is unchanged, only the order of insertions.

Everything here runs on the GPU through libwtet.so:

* ``collect``  -- training records from the plain method's own runs: the
  features of sampled vote winners of the rounds the network serves and
  whether each one inserted in its round;
* ``train``    -- the project's forward / backward / Adam kernels;
* ``loss_grad`` -- one forward + backward pass (checked against a CPU
  restatement in the tests);
* ``score``    -- the fused inference routine on given feature rows.

``make_default`` is the recipe of the packaged weights (data/learned_vote.npz).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _core

FEATURES = (
    "circumcenter_distance",   # |q - c|^2 / R^2
    "vote_score",              # log2 of the plain vote's score (circumsphere depth) / 64
    "volume_ratio",            # 6 sqrt(2) V / emax^3
    "circumradius_ratio",      # log2(R / emax) / 4
    "rival_neighbours",        # face-neighbour tets holding a vote winner / 4
    "better_rivals",           # of those winners, the ones with a larger vote score / 4
    "round",                   # log2(1 + round) / 8
    "failed_attempts",         # log2(1 + earlier vote wins without insertion) / 4
    "stratum_progress",        # uninserted points / points of the last stratum, / 2
    "round_scale",             # log2(1 + uninserted points) / 24
    "tet_size",                # -log2(emax) / 16
    "super_vertex",            # the tet has a super vertex
)
NUM_FEATURES = 12
HIDDEN = 64
NUM_PARAMS = 9217
_SHAPES = (("W1", (HIDDEN, NUM_FEATURES)), ("b1", (HIDDEN,)), ("W2", (HIDDEN, HIDDEN)), ("b2", (HIDDEN,)),
           ("W3", (HIDDEN, HIDDEN)), ("b3", (HIDDEN,)), ("W4", (HIDDEN,)), ("b4", (1,)))
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "learned_vote.npz")


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def unpack(params):
    p = np.asarray(params, np.float32)
    if p.shape != (NUM_PARAMS,):
        raise ValueError(f"expected {NUM_PARAMS} parameters, got shape {p.shape}")
    out, o = {}, 0
    for name, shape in _SHAPES:
        k = int(np.prod(shape))
        out[name] = p[o:o + k].reshape(shape)
        o += k
    return out


def pack(d):
    return np.ascontiguousarray(np.concatenate([np.asarray(d[n], np.float32).ravel() for n, _ in _SHAPES]))


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights, zero biases."""
    r = np.random.default_rng(seed)
    d = {}
    for name, shape in _SHAPES:
        if name.startswith("W"):
            fan_in = shape[-1] if len(shape) == 2 else HIDDEN
            lim = np.sqrt(6.0 / fan_in)
            d[name] = r.uniform(-lim, lim, shape)
        else:
            d[name] = np.zeros(shape)
    return pack(d)


def fold_standardization(params, mean, std):
    """Weights on raw features from weights trained on (x - mean) / std."""
    d = {k: v.astype(np.float64) for k, v in unpack(params).items()}
    w1 = d["W1"] / np.asarray(std, np.float64)[None, :]
    d["b1"] = d["b1"] - w1 @ np.asarray(mean, np.float64)
    d["W1"] = w1
    return pack(d)


def set_weights(params) -> None:
    p = np.ascontiguousarray(params, np.float32)
    L = _core.load()
    rc = L.wtet_learned_set_weights(_ptr(p), p.size)
    if rc != _core.WTET_OK:
        _core._raise(rc)


def has_weights() -> bool:
    return bool(_core.load().wtet_learned_has_weights())


def load_default(path: str = DEFAULT_WEIGHTS) -> np.ndarray:
    """Installs the packaged weights and returns them."""
    if not os.path.exists(path):
        raise FileNotFoundError(f"learned-vote weights not found at {path}; train them with "
                                "wtet_b200.learned.make_default() or install your own with set_weights()")
    with np.load(path) as z:
        params = np.ascontiguousarray(z["params"], np.float32)
    set_weights(params)
    return params


def collect(clouds, config: _core.Config | None = None, capacity: int | None = None, sample_shift: int = 0):
    """Training records (X (m, 12) float32, y (m,) uint8, stats) from the
    plain method's run on ``clouds`` (list of (N, 3) arrays): features of 1 in
    2**sample_shift of the vote winners in the rounds the learned scheduler
    serves (at most ``config.learned_gate`` x 1024 uninserted points), and
    whether each one inserted in its round (1) or not (0)."""
    arrs = [_core._points(c) for c in clouds]
    offsets = np.zeros(len(arrs) + 1, np.uint64)
    offsets[1:] = np.cumsum([a.shape[0] for a in arrs])
    pts = np.ascontiguousarray(np.concatenate(arrs, axis=0))
    n = int(offsets[-1])
    if capacity is None:
        capacity = max(1024, (8 * n) >> sample_shift)
    X = np.empty((capacity, NUM_FEATURES), np.float32)
    y = np.empty(capacity, np.uint8)
    count = ctypes.c_uint64(0)
    st = _core.Stats()
    cfg = (config or _core.Config())
    c = _core.Config(**{**cfg.__dict__, "vote": "plain"})._c()
    L = _core.load()
    rc = L.wtet_learned_collect(_ptr(pts), _ptr(offsets), len(arrs), ctypes.byref(c), int(sample_shift), _ptr(X),
                                _ptr(y), capacity, ctypes.byref(count), ctypes.byref(st))
    if rc != _core.WTET_OK:
        _core._raise(rc)
    m = count.value
    known = y[:m] != 255
    return X[:m][known].copy(), y[:m][known].copy(), st.as_dict()


def loss_grad(X, y, params):
    """(mean BCE loss, gradient) of the FP32 network, from the device kernels."""
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    p = np.ascontiguousarray(params, np.float32)
    g = np.empty(NUM_PARAMS, np.float32)
    loss = ctypes.c_float(0)
    rc = _core.load().wtet_mlp_loss_grad(_ptr(X), _ptr(y), X.shape[0], _ptr(p), ctypes.byref(loss), _ptr(g))
    if rc != _core.WTET_OK:
        _core._raise(rc)
    return float(loss.value), g


def train(X, y, params=None, epochs: int = 4, batch: int = 4096, lr: float = 2e-3, seed: int = 0,
          standardize: bool = True):
    """Trains on the device; returns (params on raw features, loss per epoch)."""
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    mean = np.zeros(NUM_FEATURES)
    std = np.ones(NUM_FEATURES)
    if standardize:
        mean = X.mean(0).astype(np.float64)
        std = X.std(0).astype(np.float64)
        std[std < 1e-6] = 1.0
        X = np.ascontiguousarray(((X - mean) / std).astype(np.float32))
    p = np.ascontiguousarray(init_params(seed) if params is None else params, np.float32).copy()
    tc = _core.TrainConfig(epochs=epochs, batch=batch, lr=lr, beta1=0.9, beta2=0.999, eps=1e-8, seed=seed)
    losses = np.zeros(max(epochs, 1), np.float32)
    rc = _core.load().wtet_mlp_train(_ptr(X), _ptr(y), X.shape[0], ctypes.byref(tc), _ptr(p), _ptr(losses))
    if rc != _core.WTET_OK:
        _core._raise(rc)
    if standardize:
        p = fold_standardization(p, mean, std)
    return p, losses[:epochs]


def score(X) -> np.ndarray:
    """Logits of the installed weights through the fused vote inference."""
    X = np.ascontiguousarray(X, np.float32)
    out = np.empty(X.shape[0], np.float32)
    rc = _core.load().wtet_mlp_score(_ptr(X), X.shape[0], _ptr(out))
    if rc != _core.WTET_OK:
        _core._raise(rc)
    return out


def training_clouds(seeds=(1, 2, 3, *range(11, 31)), size: int = 200_000):
    """The training distribution, from the small plain, degenerate and large
    plain configurations: per seed a 100k uniform cloud, a mixture cloud, a
    thin shell and a unit sphere (``size`` points, halved for the last two),
    2M-point mixture clouds from four of the seeds, 8M-point mixture clouds
    from three (the network serves the first strata, whose size grows with
    the cloud), and exact lattices of 32^3, 48^3 and 64^3 points."""
    from . import synthetic as syn

    for s in seeds:
        yield [syn.uniform(100_000, s)]
        yield [syn.mixture(size, s)]
        yield [syn.sphere_shell(size // 2, s)]
        yield [syn.unit_sphere(size // 2, s)]
    for s in seeds[3:7]:
        yield [syn.mixture(2_000_000, s)]
    for s in seeds[:3]:
        yield [syn.mixture(8_000_000, s)]
    for k in (32, 48, 64):
        yield [syn.lattice(k)]


def make_default(path: str = DEFAULT_WEIGHTS, epochs: int = 6, sample_shift: int = 3, seed: int = 0,
                 verbose: bool = True):
    """The recipe of the packaged weights: collect from the plain method's runs
    on ``training_clouds()``, train on the device, save params + metadata."""
    Xs, ys = [], []
    for clouds in training_clouds():
        X, y, _ = collect(clouds, sample_shift=sample_shift)
        Xs.append(X)
        ys.append(y)
    X = np.concatenate(Xs)
    y = np.concatenate(ys).astype(np.float32)
    r = np.random.default_rng(seed)
    idx = r.permutation(X.shape[0])
    nval = X.shape[0] // 10
    va, tr = idx[:nval], idx[nval:]
    params, losses = train(X[tr], y[tr], epochs=epochs, seed=seed)
    set_weights(params)
    s = score(X[va])
    acc = float(((s > 0) == (y[va] > 0.5)).mean())
    base = float(max(y[va].mean(), 1 - y[va].mean()))
    auc = roc_auc(s, y[va])
    if verbose:
        print(f"records {X.shape[0]} positive {y.mean():.3f} epoch losses {np.round(losses, 4).tolist()} "
              f"val acc {acc:.4f} (majority {base:.4f}) auc {auc:.3f}")
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez(path, params=params, epoch_loss=losses, val_accuracy=acc, majority=base, val_auc=auc,
             records=X.shape[0], positive_rate=float(y.mean()), sample_shift=sample_shift, seed=seed)
    return params


def roc_auc(scores, labels) -> float:
    """Area under the ROC curve of scores for binary labels (rank statistic)."""
    scores = np.asarray(scores, np.float64)
    pos = np.asarray(labels) > 0.5
    order = np.argsort(scores, kind="stable")
    ranks = np.empty(len(scores))
    ranks[order] = np.arange(1, len(scores) + 1)
    npos, nneg = int(pos.sum()), int((~pos).sum())
    if npos == 0 or nneg == 0:
        return 0.5
    return float((ranks[pos].sum() - npos * (npos + 1) / 2) / (npos * nneg))
