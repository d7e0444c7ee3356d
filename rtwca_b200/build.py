"""Builds librtw_b200.so (the CUDA trace kernels + the C ABI) in-tree for sm_100a.

Every translation unit is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a`` in parallel, then linked into
``rtwca_b200/librtw_b200.so`` (which is what the ctypes binding loads).
Runs on a machine without a GPU (nvcc cross-compiles).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "librtw_b200.so"

SOURCES = ["rtw_capi.cu", "rtw_probe.cu", "rtw_opcount.cu", "rtw_noalloc.cu", "rtw_kind0.cu", "rtw_kind1.cu", "rtw_kind2.cu", "rtw_kind3.cu", "rtw_torus.cu", "rtw_plain.cu"]
HEADERS = ["rtw_internal.h", "rtw_scenes.cuh", "rtw_trace.cuh", "rtw_launch.cuh", "rtw_ctx.h", "rtw_dual.cuh",
           "rtw_torus.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
    "-I", str(PKG.parent / "include"),
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found (CUDA toolkit required to build librtw_b200.so)")
    return cand


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: str, verbose_ptxas: bool) -> tuple[str, str]:
    obj = BUILD / (Path(src).stem + ".o")
    deps = [CSRC / src] + [CSRC / h for h in HEADERS] + [PKG.parent / "include" / "rtw.h"]
    if not _stale(obj, deps) and not verbose_ptxas:
        return src, ""
    cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else []) + ["-c", str(CSRC / src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return src, r.stderr


def build(verbose_ptxas: bool = False, jobs: int | None = None) -> Path:
    """Compile (incrementally) and link librtw_b200.so; returns its path."""
    BUILD.mkdir(exist_ok=True)
    logs = {}
    with cf.ThreadPoolExecutor(max_workers=jobs or min(len(SOURCES), os.cpu_count() or 4)) as ex:
        for src, log in ex.map(lambda s: _compile(s, verbose_ptxas), SOURCES):
            logs[src] = log
    objs = [BUILD / (Path(s).stem + ".o") for s in SOURCES]
    if _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas:
        for src, log in logs.items():
            if log:
                sys.stderr.write(f"== {src}\n{log}\n")
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv)
    print(LIB)
