"""Builds the CUDA library ``lag2d_b200/_lib/liblag2d.so`` for sm_100a with nvcc.

Two variants are built from the same sources:
  liblag2d.so        --fmad=true  (production)
  liblag2d_exact.so  --fmad=false (no FMA contraction: reproduces the CPU
                     restatement of the reference bit for bit; used by the
                     parity tests)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = [os.path.join(HERE, "csrc", f) for f in ("lag2d_kernels.cu", "lag2d_fast.cu", "lag2d_mixed.cu", "lag2d_capi.cu", "lag2d_noalloc.cu", "lag2d_p1.cu")]
OUT_DIR = os.path.join(HERE, "_lib")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _cmd(out: str, fmad: bool, extra=()):
    return [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
            f"--fmad={'true' if fmad else 'false'}", "-I", os.path.join(ROOT, "include"),
            "-cudart", "static", "-o", out, *SRC, *extra]


def targets():
    return {"liblag2d.so": True, "liblag2d_exact.so": False}


# measurement aid for bench.py (FP64 FMA peak), not part of the time-step API
BENCH_SRC = os.path.join(HERE, "csrc", "lag2d_peak.cu")
BENCH_LIB = os.path.join(OUT_DIR, "liblag2d_bench.so")


def _build_bench(verbose: bool, force: bool) -> str:
    if not force and os.path.exists(BENCH_LIB) and os.path.getmtime(BENCH_LIB) >= os.path.getmtime(BENCH_SRC):
        return BENCH_LIB
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-cudart", "static",
           "-o", BENCH_LIB, BENCH_SRC]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return BENCH_LIB


def build(verbose: bool = False, force: bool = False) -> list:
    os.makedirs(OUT_DIR, exist_ok=True)
    built = []
    deps = SRC + [os.path.join(HERE, "csrc", "lag2d_device.cuh"), os.path.join(HERE, "csrc", "lag2d_tables.inc"),
                  os.path.join(HERE, "csrc", "lag2d_fast_tables.h"), os.path.join(HERE, "csrc", "lag2d_shape9.cuh"), os.path.join(HERE, "csrc", "lag2d_p1.h"),
                  os.path.join(ROOT, "include", "lag2d.h")]
    newest = max(os.path.getmtime(p) for p in deps)
    for name, fmad in targets().items():
        out = os.path.join(OUT_DIR, name)
        if not force and os.path.exists(out) and os.path.getmtime(out) >= newest:
            built.append(out)
            continue
        cmd = _cmd(out, fmad)
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        built.append(out)
    built.append(_build_bench(verbose, force))
    return built


if __name__ == "__main__":
    for p in build(verbose=True, force="--force" in sys.argv):
        print(p)
