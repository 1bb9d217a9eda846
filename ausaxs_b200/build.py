"""Build of the sm_100a CUDA library behind the C ABI (include/ausaxs_b200.h).

Compiles every ``csrc/*.cu`` with nvcc for ``sm_100a`` only and links them into
``ausaxs_b200/_lib/libausaxs_b200.so`` (in-tree, so the built file travels with the
repository).  Incremental: a translation unit is recompiled when it or any header changed.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libausaxs_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + SRC]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build ausaxs_b200")


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(SRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, obj: str, extra: list[str]) -> str:
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    return r.stderr


SYNTH_SRC = os.path.join(SRC, "synth.c")
SYNTH_LIB = os.path.join(LIBDIR, "libsynth.so")


def build_synth(force: bool = False) -> str:
    """The seeded structure generator (plain C, host only)."""
    os.makedirs(LIBDIR, exist_ok=True)
    if force or not os.path.exists(SYNTH_LIB) or os.path.getmtime(SYNTH_LIB) < os.path.getmtime(SYNTH_SRC):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-o", SYNTH_LIB + ".tmp", SYNTH_SRC, "-lm"])
        os.replace(SYNTH_LIB + ".tmp", SYNTH_LIB)
    return SYNTH_LIB


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    """Compile (if needed) and return the path of the shared library."""
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    build_synth(force)
    srcs = sorted(glob.glob(os.path.join(SRC, "*.cu")))
    hdr = _headers_mtime()
    jobs = []
    objs = []
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or verbose_ptxas or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr):
            jobs.append((s, o))
    logs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for log in ex.map(lambda j: _compile(j[0], j[1], extra), jobs):
                logs.append(log)
    if jobs or not os.path.exists(LIB):
        tmp = LIB + ".tmp"
        cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    if verbose_ptxas:
        print("\n".join(logs))
    return LIB


if __name__ == "__main__":
    import sys

    print(build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv))
