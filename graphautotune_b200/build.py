"""Builds libgat.so (and the pm-compatible CLI) in-tree with nvcc for sm_100a.

    python -m graphautotune_b200.build [--force] [--jobs N]

Objects go to graphautotune_b200/_build/, the library to
graphautotune_b200/libgat.so and the CLI to graphautotune_b200/bin/pm.
Rebuilds only what changed (by modification time of sources and headers).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libgat.so"
CLI = PKG / "bin" / "pm"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _flags() -> list[str]:
    return [
        "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp,-O3",
        "-I", str(ROOT / "include"), "-I", str(CSRC), "--expt-relaxed-constexpr",
    ]


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.hpp")) + [ROOT / "include" / "gat.h"]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, force: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if force or _stale(obj, [src, *_headers()]):
        cmd = [nvcc(), *_flags(), "-c", str(src), "-o", str(obj)]
        if src.suffix == ".cu" and os.environ.get("GAT_PTXAS_V"):
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if os.environ.get("GAT_PTXAS_V") and r.stderr:
            sys.stderr.write(r.stderr)
    return obj


LIB_SOURCES = ["schedule.cpp", "plan.cpp", "graph.cpp", "capi.cpp", "engine.cu"]


def build(force: bool = False, jobs: int = 0) -> Path:
    BUILD.mkdir(exist_ok=True)
    (PKG / "bin").mkdir(exist_ok=True)
    srcs = [CSRC / s for s in LIB_SOURCES]
    extra = sorted(p for p in CSRC.glob("*.cu") if p.name not in LIB_SOURCES)
    srcs += extra
    jobs = jobs or min(8, os.cpu_count() or 2)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs),
               "-Xcompiler", "-fopenmp", "-lgomp", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    cli_src = CSRC / "pm_main.cpp"
    if cli_src.exists():
        cli_obj = _compile(cli_src, force)
        if force or _stale(CLI, [cli_obj, LIB]):
            cmd = [nvcc(), *ARCH, "-o", str(CLI), str(cli_obj), "-L", str(PKG), "-lgat",
                   "-Xlinker", "-rpath,$ORIGIN/..", "-lcudart"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=0)
    a = ap.parse_args()
    print(build(a.force, a.jobs))


if __name__ == "__main__":
    main()
