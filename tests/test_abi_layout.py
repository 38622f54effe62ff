"""The ctypes mirrors in wtet_b200 match the C header's struct layouts: a
small C program compiled against include/wtet.h prints sizeof / offsetof of
every public struct field, and the Python structures must agree (an ABI drift
guard for callers binding the header from other languages)."""
import ctypes
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "wtet_config": ("_core", "_Config"),
    "wtet_stats": ("_core", "Stats"),
    "wtet_train_config": ("_core", "TrainConfig"),
    "wtet_tune_entry": ("autotune", "TuneEntry"),
    "wtet_result": ("_core", "_Result"),
}


def _c_layout(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    from wtet_b200 import _core, autotune

    mods = {"_core": _core, "autotune": autotune}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "wtet.h"', "int main(void) {"]
    for cname, (mod, pyname) in STRUCTS.items():
        cls = getattr(mods[mod], pyname)
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {tuple(l.split()[:2]): int(l.split()[2]) for l in out.splitlines()}, mods


def test_struct_layouts_match_header(tmp_path):
    c, mods = _c_layout(tmp_path)
    for cname, (mod, pyname) in STRUCTS.items():
        cls = getattr(mods[mod], pyname)
        assert ctypes.sizeof(cls) == c[(cname, "size")], cname
        for field, _ in cls._fields_:
            assert getattr(cls, field).offset == c[(cname, field)], (cname, field)
