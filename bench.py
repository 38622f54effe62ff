"""Benchmark: exact 3D Delaunay throughput (Mpoints/s) on B200.

Workload (default): one cloud of 8,000,000 float32 points, a seeded mixture of
60% uniform in [0,1]^3, 30% Gaussian ball (centre 0.5, sigma 0.1) and 10% thin
spherical shell (r 0.4, radial jitter 1e-4), synthetic (numpy PCG64, seed 3).
A step = one full triangulation (normalise, sort, all insertion rounds, output
compaction).  `--workload batched` runs 4,096 clouds of log-uniform sizes in
[64, 65536] (uniform / Gaussian / shell / jittered lattice) as one step.

  value     Mpoints/s with the points already resident in HBM (device API),
            device-timed with CUDA events, max over ranks, whole job
  e2e       Mpoints/s through the C ABI (wtet_delaunay_into) from pinned host
            buffers, host->device copy of the points and device->host copy of
            tets + adjacency inside the timed region
  roofline  algorithmic bytes 12 B/point + 32 B/tet per triangulation over its
            device time, against the measured HBM copy bandwidth
  cpu_baseline  the oracle (sequential exact Bowyer-Watson restating the
            reference's CPU path) on the whole workload, 1 core; its canonical
            output is compared with the GPU's (parity)

Multi-GPU: a single cloud does not shard, so N ranks run N replicas (weak
scaling); the batched workload splits its clouds across ranks.
`--impl reference` times the reference's CPU algorithm (the oracle port; the
Rust/wgpu reference cannot be built or run on this machine) with all host
cores on the same workload and metric: each step one complete triangulation.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpoints/s on 1 B200 (exact 3D Delaunay, bit-identical tet set)"
UNIT = "Mpoints/s"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_workload(name: str, rank: int = 0, world: int = 1):
    from wtet_b200 import synthetic as syn

    if name == "mixture8M":
        return [syn.mixture(8_000_000, 3)]
    if name == "mixture8M_new":
        return [syn.mixture(8_000_000, 101)]
    if name == "mixture1M":
        return [syn.mixture(1_000_000, 3)]
    if name == "mixture100k":
        return [syn.mixture(100_000, 3)]
    if name == "lattice2M":
        return [syn.lattice(128)]
    if name == "sphere1M":
        return [syn.unit_sphere(1_000_000, 2)]
    if name == "uniform8M":
        return [syn.uniform(8_000_000, 1)]
    if name == "uniform100k":
        return [syn.uniform(100_000, 1)]
    if name == "batched":
        return shard(syn.batched_clouds(4096, 4), rank, world)
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus, backend: str = "nccl"):
    """One process per GPU (torchrun env); a short process-group timeout so
    that ranks waiting on a dead peer end with an error."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return rank, local, world


def reduce_over_ranks(x: float, world: int, op: str = "max", device: str = "cuda") -> float:
    """max / sum of a scalar over all ranks (the same value on every rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float, world: int) -> float:
    return reduce_over_ranks(x, world, "max")


def cloud_cost(n: int) -> float:
    """Estimated work of one cloud: n log n (point location and the rounds
    of a cloud grow like that)."""
    return float(n) * np.log2(max(int(n), 2))


def lpt_assign(sizes, world: int):
    """Longest-processing-time-first assignment of clouds to ranks: clouds in
    decreasing estimated cost, each to the rank with the least work so far.
    Returns the rank of every cloud (deterministic: ties go to the lower
    rank, equal costs keep their input order)."""
    order = sorted(range(len(sizes)), key=lambda i: (-cloud_cost(sizes[i]), i))
    load = [0.0] * world
    owner = [0] * len(sizes)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += cloud_cost(sizes[i])
    return owner


def shard(clouds, rank: int, world: int):
    """Clouds of a batched workload owned by one rank (LPT over the n log n
    cost estimate, input order kept inside a rank); a single cloud is not
    split -- every rank runs a replica."""
    if len(clouds) == 1 or world == 1:
        return clouds
    owner = lpt_assign([len(c) for c in clouds], world)
    return [c for c, o in zip(clouds, owner) if o == rank]


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def bench_config(workload: str, vote: str, world: int):
    """The workload description printed by both arms (identical dicts, so the
    two lines are on the same configuration)."""
    clouds = 1 if workload != "batched" else 4096
    cfg = {
        "workload": workload,
        "description": WORKLOADS[workload],
        "points": POINTS[workload],
        "clouds": clouds,
        "vote": vote,
        "parallelism": "replicas (a single triangulation does not shard)" if clouds == 1
        else "clouds split across ranks by LPT over n log n, no data-path collective",
        "l2": "inputs larger than the 126 MB L2: tets, adjacency and claim arrays of several GB",
    }
    if workload == "batched":
        cfg["batching"] = "all clouds in one job: insertion rounds over every cloud replayed from CUDA graphs " \
                          "(graph nodes are the grid-wide barriers; no persistent kernel)"
    return cfg


def run_gpu(args):
    import torch

    import wtet_b200 as wt

    rank, local, world = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    wt._core.load()
    L = wt._core.load()
    clouds = make_workload(args.workload, rank, world)
    n_points = sum(len(c) for c in clouds)
    cfg = wt.Config(vote=args.vote)._c()

    # ---- device-resident arm: points in HBM, output buffers preallocated ----
    stream = torch.cuda.current_stream()
    if len(clouds) == 1:
        d_pts = torch.from_numpy(clouds[0]).cuda()
        cap = int(L.wtet_max_tets(n_points))
        d_t = torch.empty((cap, 4), dtype=torch.int32, device="cuda")
        d_a = torch.empty((cap, 4), dtype=torch.int32, device="cuda")
        m = ctypes.c_uint64(0)
        st = wt._core.Stats()

        def step():
            rc = L.wtet_delaunay_device(ctypes.c_void_p(d_pts.data_ptr()), n_points, ctypes.byref(cfg),
                                        ctypes.c_void_p(d_t.data_ptr()), ctypes.c_void_p(d_a.data_ptr()), cap,
                                        ctypes.byref(m), ctypes.byref(st), ctypes.c_void_p(stream.cuda_stream))
            if rc != 0:
                raise RuntimeError(L.wtet_last_error().decode())
            return m.value, st
    else:
        pts = np.ascontiguousarray(np.concatenate(clouds))
        offsets = np.zeros(len(clouds) + 1, np.uint64)
        offsets[1:] = np.cumsum([len(c) for c in clouds])
        cap = int(sum(int(L.wtet_max_tets(len(c))) for c in clouds))
        h_t = torch.empty((cap, 4), dtype=torch.int32, pin_memory=True)
        h_a = torch.empty((cap, 4), dtype=torch.int32, pin_memory=True)
        toff = np.zeros(len(clouds) + 1, np.uint64)
        st = wt._core.Stats()
        h_pts = torch.from_numpy(pts).pin_memory()

        def step():
            rc = L.wtet_delaunay_batched(ctypes.c_void_p(h_pts.data_ptr()), ctypes.c_void_p(offsets.ctypes.data),
                                         len(clouds), ctypes.byref(cfg), ctypes.c_void_p(h_t.data_ptr()),
                                         ctypes.c_void_p(h_a.data_ptr()), cap, ctypes.c_void_p(toff.ctypes.data),
                                         ctypes.byref(st))
            if rc != 0:
                raise RuntimeError(L.wtet_last_error().decode())
            return int(toff[-1]), st

    if args.profile_once:
        # one triangulation and nothing else: a short, complete launch list for ncu
        num, s = step()
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"profile_once": args.workload, "num_tets": num, "rounds": s.rounds,
                              "kernel_launches": s.kernel_launches, "device_ms": s.device_ms}))
        return
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    dev_ms, launches, rounds, num_tets = [], 0, 0, 0
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            num_tets, s = step()
            dev_ms.append(s.device_ms)
            launches += s.kernel_launches
            rounds = s.rounds
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    elapsed_ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    ms_step = elapsed_ms / args.steps
    total_points = n_points * (world if len(clouds) == 1 else 1)
    if len(clouds) > 1 and world > 1:
        total_points = int(reduce_over_ranks(float(n_points), world, "sum"))
    value = total_points / (ms_step * 1e3)

    # ---- end-to-end arm: C ABI from pinned host buffers, copies inside ----
    e2e = None
    if len(clouds) == 1:
        h_pts = torch.from_numpy(clouds[0]).pin_memory()
        h_t = torch.empty((cap, 4), dtype=torch.int32, pin_memory=True)
        h_a = torch.empty((cap, 4), dtype=torch.int32, pin_memory=True)
        failed = np.empty(n_points, np.uint32)
        st2 = wt._core.Stats()
        m2 = ctypes.c_uint64(0)

        def step_e2e():
            rc = L.wtet_delaunay_into(ctypes.c_void_p(h_pts.data_ptr()), n_points, ctypes.byref(cfg),
                                      ctypes.c_void_p(h_t.data_ptr()), ctypes.c_void_p(h_a.data_ptr()), cap,
                                      ctypes.byref(m2), ctypes.c_void_p(failed.ctypes.data), ctypes.byref(st2))
            if rc != 0:
                raise RuntimeError(L.wtet_last_error().decode())

        step_e2e()
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(max(1, args.steps)):
            step_e2e()
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / max(1, args.steps), world)
        e2e = {"value": round(total_points / (e2e_ms * 1e3), 4), "unit": UNIT,
               "h2d_bytes_per_step": int(12 * n_points), "d2h_bytes_per_step": int(32 * m2.value),
               "ms_per_step": round(e2e_ms, 3)}
    else:
        e2e = {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": int(12 * n_points),
               "d2h_bytes_per_step": int(32 * num_tets), "ms_per_step": round(ms_step, 3),
               "note": "the batched step already runs through the C ABI from pinned host buffers"}

    hbm, peak_kind = peaks()
    per_run_ms = float(np.mean(dev_ms))
    alg_bytes = 12 * n_points + 32 * num_tets
    achieved = alg_bytes / (per_run_ms * 1e-3) / 1e9
    result = {
        "metric": METRIC,
        "value": round(value, 4),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": bench_config(args.workload, args.vote, world),
        "e2e": e2e,
        "gpu_launches": int(launches),
        "rounds": int(rounds),
        "num_tets": int(num_tets),
        "roofline": {
            "bound": "hbm",
            "achieved": round(achieved, 2),
            "peak": hbm,
            "unit": "GB/s",
            "frac": round(achieved / hbm, 5),
            "traffic": TRAFFIC.get(args.workload),
            "traffic_source": TRAFFIC_SOURCE if args.workload in TRAFFIC else None,
            "basis": "whole triangulation per step (thousands of launches of the round kernels replayed from "
                     "CUDA graphs, so no single launch is the unit): 12 B/point read + 32 B/tet written over its "
                     f"device time; peak = {peak_kind} copy bandwidth; traffic = DRAM bytes read + written by all "
                     "launches of one triangulation (ncu)",
        },
        "clocks": clocks.summary(),
    }
    golden = golden_digests()
    if len(clouds) == 1:
        # the last step's output, canonical on the device, against the oracle's
        gdig = device_digest(wt, d_t, d_a, num_tets, n_points)
        gname = GOLDEN_NAME.get(args.workload)
        result["parity"] = {"canonical_sha256": gdig,
                            "same_as_stored_oracle_digest": bool(gname in golden and golden[gname]["sha256"] == gdig)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline and len(clouds) == 1:
        result["cpu_baseline"] = cpu_baseline(clouds[0], result["parity"]["canonical_sha256"])
    if world == 1 and args.variants and args.workload == "mixture8M" and args.vote == "plain":
        result["variants"] = variants(wt, args, golden)
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# DRAM bytes (read + write) of one whole triangulation of the 8M mixture,
# estimated with ncu: for each round kernel, the DRAM bytes per microsecond of
# one launch in the most expensive round of the 1M mixture (one kernel, one
# launch per capture) times that kernel's total time in the time-only launch
# list of one 8M triangulation.  It describes the kernels it was measured on
# and must be captured again when they change.
TRAFFIC: dict = {"mixture8M": 366.7e9}
TRAFFIC_SOURCE = ("estimate: sum over k_bfs, k_shared, k_write, k_cands, k_relocate, k_activate of "
                  "(DRAM bytes per us of one bulk-round launch on the 1M mixture, ncu) x (the kernel's total time "
                  "in the 8M launch list, ncu); early rounds fit in L2, so this over-counts them; two captures of "
                  "different bulk rounds gave 312 and 367 GB")

WORKLOADS = {
    "mixture8M": "8,000,000 points: 60% uniform [0,1]^3, 30% Gaussian ball (0.5, sigma 0.1), "
                 "10% thin shell r=0.4 (jitter 1e-4); float32, seed 3",
    "uniform8M": "8,000,000 points uniform in [0,1]^3, float32, seed 1",
    "mixture8M_new": "the 8M mixture's distribution from a seed no training run saw (seed 101)",
    "mixture1M": "1,000,000 points of the 8M mixture's distribution (profiling size)",
    "uniform100k": "100,000 points uniform in [0,1]^3, float32, seed 1 (the small plain configuration)",
    "mixture100k": "100,000 points of the 8M mixture's distribution (profiling size)",
    "lattice2M": "128^3 = 2,097,152 points on the exact lattice float32(i)/127 (SoS stress)",
    "sphere1M": "1,000,000 points on the unit sphere (normalised Gaussian directions), float32, seed 2",
    "batched": "4,096 clouds, sizes log-uniform in [64, 65536], each uniform / Gaussian / shell / "
               "jittered lattice, float32, seed 4",
}
POINTS = {"mixture8M": 8_000_000, "uniform8M": 8_000_000, "mixture8M_new": 8_000_000, "mixture1M": 1_000_000,
          "uniform100k": 100_000, "mixture100k": 100_000, "lattice2M": 128 ** 3, "sphere1M": 1_000_000,
          "batched": 39_908_171}
# workload -> entry of tests/golden/full_size.json (the oracle's canonical digest)
GOLDEN_NAME = {"mixture8M": "mixture8M_s3", "mixture8M_new": "mixture8M_s101", "lattice2M": "lattice128",
               "sphere1M": "unit_sphere1M", "uniform100k": "uniform100k"}


def golden_digests():
    p = os.path.join(ROOT, "tests", "golden", "full_size.json")
    if not os.path.exists(p):
        return {}
    with open(p) as f:
        return json.load(f)


def device_digest(wt, d_t, d_a, m, n):
    """Canonical form of the first m output rows on the device, as SHA-256."""
    ct, ca = wt.canonical_device(d_t[:m], d_a[:m], n)
    return wt.canonical_digest(ct, ca)


def device_run(wt, L, d_pts, n, cfg, d_t, d_a, cap, stream):
    m = ctypes.c_uint64(0)
    st = wt._core.Stats()
    rc = L.wtet_delaunay_device(ctypes.c_void_p(d_pts.data_ptr()), n, ctypes.byref(cfg),
                                ctypes.c_void_p(d_t.data_ptr()), ctypes.c_void_p(d_a.data_ptr()), cap,
                                ctypes.byref(m), ctypes.byref(st), ctypes.c_void_p(stream.cuda_stream))
    if rc != 0:
        raise RuntimeError(L.wtet_last_error().decode())
    return m.value, st


def variants(wt, args, golden):
    """The metric's other two forms, each on its own configuration, device
    time (CUDA events inside the library), each output compared with the
    oracle's stored canonical digest:
      learned  8M mixture clouds from seeds 101-105 (no training run saw them),
               plain vs learned scheduler;
      learned_lattice  the 128^3 lattice, plain vs learned;
      batched  4,096 clouds in one call vs looping the plain path over them."""
    import torch

    from wtet_b200 import synthetic as syn

    L = wt._core.load()
    stream = torch.cuda.current_stream()
    reps = 5
    out = {}

    def compare(pts, gname):
        """Plain and learned on the same cloud: one warm-up each, then reps
        runs of each, alternating, so that a slow period of the shared host
        or GPU affects both; median device time of each."""
        n = len(pts)
        d_pts = torch.from_numpy(pts).cuda()
        cap = int(L.wtet_max_tets(n))
        votes = ("plain", "learned")
        bufs = {v: (torch.empty((cap, 4), dtype=torch.int32, device="cuda"),
                    torch.empty((cap, 4), dtype=torch.int32, device="cuda")) for v in votes}
        cfgs = {v: wt.Config(vote=v)._c() for v in votes}
        for v in votes:
            device_run(wt, L, d_pts, n, cfgs[v], *bufs[v], cap, stream)
        runs = {v: [] for v in votes}
        for _ in range(reps):
            for v in votes:
                runs[v].append(device_run(wt, L, d_pts, n, cfgs[v], *bufs[v], cap, stream))
        recs = {}
        for v in votes:
            m, st = runs[v][-1]
            dig = device_digest(wt, *bufs[v], m, n)
            ms = float(np.median([r[1].device_ms for r in runs[v]]))
            recs[v] = {"mpts": round(n / (ms * 1e3), 3), "device_ms": round(ms, 2), "rounds": int(st.rounds),
                       "vote_winners": int(st.vote_winners), "cavity_searches": int(st.candidates),
                       "same_as_oracle": bool(gname in golden and dig == golden[gname]["sha256"])}
        del bufs, d_pts
        torch.cuda.empty_cache()
        return recs

    seeds = []
    for seed in range(101, 106):
        rec = {"seed": seed}
        for vote, r in compare(syn.mixture(8_000_000, seed), f"mixture8M_s{seed}").items():
            for k, v in r.items():
                rec[f"{vote}_{k}"] = v
        seeds.append(rec)
    out["learned"] = {
        "workload": "8,000,000-point mixture clouds, seeds 101-105",
        "how": f"per seed: one warm-up each, then {reps} runs of each scheduler alternating; median device time",
        "per_seed": seeds,
        "plain_mpts_mean": round(float(np.mean([r["plain_mpts"] for r in seeds])), 3),
        "learned_mpts_mean": round(float(np.mean([r["learned_mpts"] for r in seeds])), 3),
        "learned_faster_on": sum(r["learned_mpts"] > r["plain_mpts"] for r in seeds),
        "all_same_as_oracle": all(r["plain_same_as_oracle"] and r["learned_same_as_oracle"] for r in seeds),
    }
    out["learned_lattice"] = {"workload": "lattice2M",
                              **{f"{v}_{k}": x for v, r in compare(syn.lattice(128), "lattice128").items()
                                 for k, x in r.items()}}
    clouds = make_workload("batched")
    n = sum(len(c) for c in clouds)
    wt.delaunay_batched(clouds)
    bms = []
    for _ in range(reps):
        rb = wt.delaunay_batched(clouds)
        bms.append(rb[0].stats["device_ms"])
    same_b = True
    gb = os.path.join(ROOT, "tests", "golden", "batched_digests.npz")
    if os.path.exists(gb):
        want = np.load(gb)["digests"]
        for i, (c, r) in enumerate(zip(clouds, rb)):
            ct, ca = wt.canonical(r.tets, r.adjacency, len(c))
            same_b = same_b and bytes.fromhex(wt.canonical_digest(ct, ca)) == want[i].tobytes()
    else:
        same_b = None
    loop_ms = 0.0
    for c in clouds:
        loop_ms += wt.delaunay(c).stats["device_ms"]
    bm = float(np.median(bms))
    out["batched"] = {"workload": "batched", "clouds": len(clouds), "points": n, "all_same_as_oracle": same_b,
                      "batched_mpts": round(n / (bm * 1e3), 3), "batched_device_ms": round(bm, 1),
                      "looped_plain_mpts": round(n / (loop_ms * 1e3), 3), "looped_device_ms": round(loop_ms, 1),
                      "how": "one job over all clouds, insertion rounds replayed from CUDA graphs (no persistent "
                             "kernel: consecutive graph nodes are the grid-wide barriers)"}
    return out


def cpu_baseline(points, gpu_digest):
    """The oracle (the reference's exact Bowyer-Watson, src/phase2.rs:383-606,
    restated with walk point location) on the whole workload, one core; its
    canonical output is compared with the GPU's."""
    import oracle

    oracle.build()
    pts = np.ascontiguousarray(points)
    t0 = time.perf_counter()
    tets, adj, _ = oracle.delaunay(pts, 1)
    dt = time.perf_counter() - t0
    od = oracle.digest(*oracle.canonical(tets, adj, len(pts)))
    return {"value": round(len(pts) / dt / 1e6, 4), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"the whole workload ({len(pts)} points), one oracle triangulation on one core ({dt:.1f} s)",
            "host_cpu": host_cpu(), "oracle_digest": od, "gpu_output_identical": od == gpu_digest}


def host_cpu():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip() + f" x{os.cpu_count()}"
    except Exception:
        pass
    return f"{os.cpu_count()} cpus"


def host_memory_available():
    """Bytes of host memory available now (MemAvailable), or None."""
    try:
        with open("/proc/meminfo") as f:
            for ln in f:
                if ln.startswith("MemAvailable:"):
                    return int(ln.split()[1]) * 1024
    except Exception:
        pass
    return None


def run_reference(args):
    """CPU reference arm: the reference's CPU algorithm (the oracle port of
    src/phase2.rs:383-606 with walk point location; the Rust/wgpu reference
    cannot be built or run here) on every host core (as many at once as host
    memory holds).  A step is one complete triangulation of the same workload
    as the GPU arm; the threads take steps from a queue (W untimed warm-up
    steps first, then exactly K timed steps)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import concurrent.futures as cf

    import oracle

    oracle.build()
    clouds = make_workload(args.workload)
    threads = max(1, os.cpu_count() or 1)
    # Concurrent triangulations are bounded by host memory as well: one
    # oracle triangulation holds about 540 B per point at its peak (4.3 GB
    # for the 8M mixture); 600 B per point and 80% of the available memory
    # leave a margin.
    avail = host_memory_available()
    if avail:
        per_run = 600 * max(len(c) for c in clouds)
        threads = max(1, min(threads, int(0.8 * avail) // per_run))

    def one_step():
        for c in clouds:
            oracle.triangulate_count(c, 1)

    def run_steps(k):
        if k <= 0:
            return
        with cf.ThreadPoolExecutor(min(threads, k)) as ex:
            list(ex.map(lambda _: one_step(), range(k)))

    run_steps(args.warmup)
    t0 = time.perf_counter()
    run_steps(args.steps)
    ms = (time.perf_counter() - t0) * 1e3 / args.steps
    npts = sum(len(c) for c in clouds)
    v = npts / (ms * 1e3)
    desc = (f"{args.steps} complete triangulations of the workload ({npts} points each), "
            f"up to {min(threads, args.steps)} at a time on {threads} threads")
    out = {"impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": bench_config(args.workload, args.vote, 1),
           "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": threads, "kind": "port", "sample": desc,
                            "host_cpu": host_cpu()},
           "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "note": "the reference's CPU algorithm restated (oracle/); its Rust + wgpu path cannot be built "
                   "or run on this machine"}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="wtet_b200", choices=["wtet_b200", "reference"])
    ap.add_argument("--workload", default="mixture8M", choices=sorted(WORKLOADS))
    ap.add_argument("--vote", default="plain", choices=["plain", "learned"])
    ap.add_argument("--no-variants", dest="variants", action="store_false",
                    help="skip the learned-scheduler and batched measurements")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-once", action="store_true",
                    help="run a single triangulation and exit (for ncu launch lists)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
