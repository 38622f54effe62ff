"""The benchmark's JSON contract, on the CPU: the reference arm (the
reference's CPU algorithm, restated in oracle/) prints one line with the
metric, unit, config, cpu_baseline and e2e keys, on the same configuration as
the GPU arm, and bounds its concurrency by host memory."""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "uniform100k", "--steps", "2", "--warmup", "1"], capture_output=True, text=True,
                         timeout=600, check=True).stdout
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "dtype", "data", "config", "cpu_baseline", "e2e", "impl"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["config"] == bench.bench_config("uniform100k", "plain", 1)  # the GPU arm's config
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == d["value"] and 1 <= cb["cores"] <= (os.cpu_count() or 1)


def test_host_memory_reading():
    avail = bench.host_memory_available()
    assert avail is None or avail > 0


def test_workload_sizes_match_their_descriptions():
    for name in ("uniform100k", "mixture100k", "sphere1M", "lattice2M"):
        clouds = bench.make_workload(name)
        assert sum(len(c) for c in clouds) == bench.POINTS[name]
    assert set(bench.GOLDEN_NAME) <= set(bench.WORKLOADS)
