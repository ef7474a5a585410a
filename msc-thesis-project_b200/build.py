"""Builds libflsgpu_b200.so in-tree from csrc/*.cu for sm_100a.

    python msc-thesis-project_b200/build.py [-j N] [--force]

Each translation unit is compiled to an object under _build/ (skipped when
up to date) and linked into msc-thesis-project_b200/libflsgpu_b200.so with
the CUDA runtime linked statically."""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libflsgpu_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills", "-diag-suppress", "177,550"]


_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(path: Path, seen: set[Path] | None = None) -> set[Path]:
    """The file and every local header it includes, recursively."""
    seen = seen if seen is not None else set()
    path = path.resolve()
    if path in seen or not path.exists():
        return seen
    seen.add(path)
    for inc in _INCLUDE.findall(path.read_text()):
        _deps(path.parent / inc, seen)
    return seen


def compile_one(src: Path, force: bool, extra: list[str]) -> Path:
    obj = BUILD / (src.stem + ".o")
    newest = max(p.stat().st_mtime for p in _deps(src))
    if force or not obj.exists() or obj.stat().st_mtime < newest:
        cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src.name}")
        if r.stderr.strip():
            sys.stderr.write(f"[{src.name}]\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int = 8, extra: list[str] | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force, extra or []), srcs))
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcuda"]
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/smem usage")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_v else []
    print(build(a.force or a.ptxas_v, a.j, extra))
