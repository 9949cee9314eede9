"""Build libbsn.so (sm_100a) in-tree from csrc/*.cu with nvcc.

Usage: python build_lib.py [--force] [--verbose]

Every translation unit is compiled for sm_100a only.  The FP64 parity path
(files listed in FP64_PARITY) is compiled with -fmad=false so that no
multiply-add is contracted and results match the reference's CPU arithmetic
bit for bit; the FP32 stencil units are built the same way with their
multiply-adds written out, the FP32 FFTs keep contraction on.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OUT = os.path.join(HERE, "bsn", "libbsn.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BASE = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC]
FP64_PARITY = {"hydro_f64.cu", "sources_f64.cu", "fmr_f64.cu", "fmr_nlevel.cu", "poisson.cu", "context.cu", "cfl_noalloc.cu",
               "run_steps.cu", "autotune.cu", "coupled_run.cu", "diagnostics.cu", "relax.cu", "tma_host.cu"}
# the FP32 fast path: approximate division and square root.  The stencil
# units write every multiply-add out (fmaf, fma.rn.f32x2) and are built
# without contraction, so their results do not depend on the compiler's
# contraction choices (each tile variant gives the same bits); the FP32 FFTs
# keep contraction on.
FAST = {"stage_fast.cu", "learned.cu", "poisson_f32.cu"}
FAST_FLAGS = ["--ftz=true", "--prec-div=false", "--prec-sqrt=false", "--fmad=true"]
EXPLICIT_FMA = {"stage_fast.cu", "learned.cu"}


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps_mtime():
    return max(os.path.getmtime(os.path.join(CSRC, f)) for f in os.listdir(CSRC)
               if f.endswith((".cuh", ".h"))) if any(f.endswith((".cuh", ".h")) for f in os.listdir(CSRC)) else 0


def _compile(src: str, force: bool, verbose: bool):
    obj = os.path.join(OBJ, src[:-3] + ".o")
    srcp = os.path.join(CSRC, src)
    hdr = max(_deps_mtime(), os.path.getmtime(os.path.join(INCLUDE, "bsn.h")))
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(srcp), hdr):
        return obj, None
    flags = list(BASE)
    if src in FP64_PARITY:
        flags += ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"]
    elif src in FAST:
        flags += FAST_FLAGS
        if src in EXPLICIT_FMA:
            flags[-1] = "--fmad=false"
    cmd = [NVCC] + ARCH + flags + ["-c", srcp, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, (r.stderr if verbose else None)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for (o, log), s in zip(results, srcs):
            if log:
                print(f"== {s}\n{log}")
    if force or not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
