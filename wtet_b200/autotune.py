"""Autotuner: measures the fastest performance knobs per size bucket and
persists them as a table that the library applies to every job whose knobs
are left at 0 (``Config`` defaults).

Knobs (none changes the triangulation, which the tuner verifies):
  block_size        threads per block of the per-point kernels (128/256/512)
  rounds_per_graph  insertion rounds per CUDA-graph launch (4..32)
  overlap_shift     when the next stratum starts (the current one thinned to 1/2^k)
  candidate_filter  neighbourhood pre-claim before cavity growth (1 on, 2 off)
  pool_factor       cavity-pool entries per point (the round's candidate queue)

Buckets are by total points and by job kind (one cloud / a batch of clouds).
Each bucket is tuned by coordinate descent on a seeded synthetic workload of
its size (device time, median of ``repeats`` runs).  ``python -m
wtet_b200.autotune --out FILE`` writes a table; ``load(FILE)`` installs one;
the package installs ``data/autotune.json`` when it loads the library.
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import os
import time

import numpy as np

from . import _core

DEFAULT_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "autotune.json")
KNOBS = ("overlap_shift", "rounds_per_graph", "block_size", "candidate_filter", "pool_factor")
CHOICES = {
    "overlap_shift": (2, 3, 4, 5),
    "rounds_per_graph": (4, 8, 16, 32),
    "block_size": (128, 256, 512),
    "candidate_filter": (1, 2),
    "pool_factor": (12, 24, 48),
}
DEFAULTS = {"overlap_shift": 3, "rounds_per_graph": 8, "block_size": 256, "candidate_filter": 1, "pool_factor": 24}
# (kind, max_points, workload used to tune the bucket)
BUCKETS = (
    (0, 1 << 15, ("mixture", 20_000)),
    (0, 1 << 18, ("mixture", 200_000)),
    (0, 1 << 21, ("mixture", 1_000_000)),
    (0, 1 << 23, ("mixture", 4_000_000)),
    (0, (1 << 64) - 1, ("mixture", 8_000_000)),
    (1, 1 << 22, ("batched", 256)),
    (1, (1 << 64) - 1, ("batched", 1024)),
)


class TuneEntry(ctypes.Structure):
    _fields_ = [
        ("max_points", ctypes.c_uint64),
        ("batched", ctypes.c_uint32),
        ("block_size", ctypes.c_uint32),
        ("rounds_per_graph", ctypes.c_uint32),
        ("overlap_shift", ctypes.c_uint32),
        ("candidate_filter", ctypes.c_uint32),
        ("pool_factor", ctypes.c_uint32),
    ]


def install(table) -> None:
    """Installs a table (list of dicts with max_points, batched and knobs)."""
    L = _core.load()
    arr = (TuneEntry * max(len(table), 1))()
    for i, e in enumerate(table):
        arr[i].max_points = int(e["max_points"])
        arr[i].batched = int(e["batched"])
        for k in KNOBS:
            setattr(arr[i], k, int(e.get(k, 0)))
    rc = L.wtet_autotune_set_table(arr, len(table))
    if rc != _core.WTET_OK:
        _core._raise(rc)


def installed():
    L = _core.load()
    n = ctypes.c_uint32(0)
    L.wtet_autotune_get_table(None, 0, ctypes.byref(n))
    arr = (TuneEntry * max(n.value, 1))()
    L.wtet_autotune_get_table(arr, n.value, ctypes.byref(n))
    return [{k: int(getattr(arr[i], k)) for k, _ in TuneEntry._fields_} for i in range(n.value)]


def resolve(n: int, num_clouds: int = 1, config: _core.Config | None = None) -> dict:
    """The knobs a job of n points in num_clouds clouds runs with."""
    L = _core.load()
    out = _core._Config()
    c = (config or _core.Config())._c()
    rc = L.wtet_autotune_resolve(ctypes.byref(c), int(n), int(num_clouds), ctypes.byref(out))
    if rc != _core.WTET_OK:
        _core._raise(rc)
    return {k: int(getattr(out, k)) for k in KNOBS}


def load(path: str = DEFAULT_TABLE) -> list:
    with open(path) as f:
        table = json.load(f)["table"]
    install(table)
    return table


def save(table, path: str, meta=None) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump({"table": table, "meta": meta or {}}, f, indent=1)


def _workload(spec, seed=7):
    from . import synthetic as syn

    kind, size = spec
    if kind == "mixture":
        return [syn.mixture(size, seed)]
    return syn.batched_clouds(size, seed)


def tet_set_digest(tets) -> str:
    """Order-independent digest of a tet set: each tet's sorted vertex ids
    are mixed into a 64-bit value and the values summed (mod 2^64), so no
    sort of the whole set is needed."""
    t = np.sort(np.asarray(tets).astype(np.uint64), axis=1)
    h = t[:, 0] * np.uint64(0x9E3779B97F4A7C15)
    for k, c in ((1, 0xBF58476D1CE4E5B9), (2, 0x94D049BB133111EB), (3, 0xD6E8FEB86659FD93)):
        h = (h ^ (h >> np.uint64(29))) * np.uint64(c) + t[:, k]
    h = h ^ (h >> np.uint64(32))
    return f"{int(h.sum(dtype=np.uint64)):016x}:{t.shape[0]}"


def _digest(results) -> str:
    return "|".join(tet_set_digest(r.tets) for r in results) if len(results) < 8 else \
        tet_set_digest(np.concatenate([r.tets for r in results]))


def _measure(clouds, knobs, repeats):
    cfg = _core.Config(**knobs)
    times, dig = [], None
    for _ in range(repeats):
        if len(clouds) == 1:
            res = [_core.delaunay(clouds[0], cfg)]
        else:
            res = _core.delaunay_batched(clouds, cfg)
        times.append(res[0].stats["device_ms"])
        dig = dig or _digest(res)
    return float(np.median(times)), dig


def tune_bucket(clouds, repeats: int = 3, verbose: bool = True) -> dict:
    """Coordinate descent over KNOBS from the defaults; every choice must give
    the same tet set as the defaults."""
    best = dict(DEFAULTS)
    _measure(clouds, best, 1)  # warm-up (allocations, graph capture)
    best_ms, ref = _measure(clouds, best, repeats)
    for k in KNOBS:
        for v in CHOICES[k]:
            if v == best[k]:
                continue
            trial = {**best, k: v}
            ms, dig = _measure(clouds, trial, repeats)
            if dig != ref:
                raise RuntimeError(f"knob {k}={v} changed the triangulation")
            if verbose:
                print(f"  {k}={v}: {ms:.2f} ms (best {best_ms:.2f})", flush=True)
            if ms < best_ms * 0.98:
                best, best_ms = trial, ms
    return {**best, "device_ms": best_ms}


def tune(buckets=BUCKETS, repeats: int = 3, verbose: bool = True):
    table = []
    for kind, max_points, spec in buckets:
        clouds = _workload(spec)
        t0 = time.time()
        if verbose:
            print(f"bucket kind={kind} max_points={max_points} workload={spec}", flush=True)
        r = tune_bucket(clouds, repeats, verbose)
        if verbose:
            print(f"  -> {r} ({time.time() - t0:.1f} s)", flush=True)
        table.append({"max_points": int(max_points), "batched": kind, **{k: r[k] for k in KNOBS},
                      "device_ms": r["device_ms"], "workload": list(spec)})
    return table


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--quick", action="store_true", help="only the buckets up to 1M points")
    a = ap.parse_args(argv)
    buckets = [b for b in BUCKETS if not a.quick or (b[2][0] == "mixture" and b[2][1] <= 1_000_000)]
    install([])  # measure from the built-in defaults
    table = tune(buckets, a.repeats)
    save(table, a.out, {"gpu": _core.gpu_info(), "repeats": a.repeats})
    install(table)
    print(json.dumps(table, indent=1))


if __name__ == "__main__":
    main()
