"""Static check of the CUDA sources: every kernel declared with
__launch_bounds__(max_threads, ...) is launched with a block size that can
never exceed max_threads.  A launch beyond the bound fails at run time (and,
inside a stream capture, fails the whole graph); block sizes come from a
literal or from TB, the per-point block size the configuration may set to
128, 256 or 512."""
import os
import re

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "wtet_b200", "csrc")
TB_MAX = 512  # cfg.block_size is clamped to 128 / 256 / 512


def _sources():
    for name in sorted(os.listdir(CSRC)):
        if name.endswith(".cu"):
            with open(os.path.join(CSRC, name)) as f:
                yield name, f.read()


def test_launch_bounds_are_respected():
    checked = 0
    for name, src in _sources():
        bounds = {m.group(2): int(m.group(1))
                  for m in re.finditer(r"__launch_bounds__\((\d+)[^)]*\)\s+(\w+)\s*\(", src)}
        for m in re.finditer(r"\b(\w+)<<<\s*[^,]+,\s*([^,>]+?)\s*(?:,[^>]*)?>>>", src):
            kernel, block = m.group(1), m.group(2).strip()
            if kernel not in bounds:
                continue
            if block.isdigit():
                size = int(block)
            elif block == "TB":
                size = TB_MAX
            else:
                raise AssertionError(f"{name}: cannot size the launch of {kernel} with block '{block}'")
            assert size <= bounds[kernel], f"{name}: {kernel} launched with up to {size} > bound {bounds[kernel]}"
            checked += 1
    assert checked >= 5
