"""Build recipe of the in-tree native libraries.

* ``libampcor_b200.so`` - the sm_100a kernels and the C ABI (nvcc, ``-gencode
  arch=compute_100a,code=sm_100a``), with the CUDA runtime linked statically;
* ``libampcor_synth.so`` - the host-side raster warper used to synthesise benchmark inputs;
* ``libampcor_peak.so`` - an FP32 FMA throughput probe (the SIMT roofline the benchmark
  reports the plain form against).

Run ``python -m ampcor_b200.build`` (``--force`` to rebuild).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CC = "/usr/bin/gcc"

CUDA_SOURCES = ["kernels.cu", "tc_ncc.cu", "tc_zoom.cu", "spectral.cu", "capi.cu"]
CUDA_HEADERS = ["kernels.cuh", "tile_common.cuh", "fft.cuh", "tcgen05.cuh", os.path.join("..", "..", "include", "ampcor_b200.h")]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared", "-Xlinker", "--no-undefined",
]

LIB = os.path.join(HERE, "libampcor_b200.so")
SYNTH = os.path.join(HERE, "libampcor_synth.so")
PEAK = os.path.join(HERE, "libampcor_peak.so")


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(force: bool = False, verbose: bool = False) -> None:
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in CUDA_HEADERS]
    if force or _stale(LIB, deps):
        cmd = [NVCC, *NVCC_FLAGS, "-o", LIB, *srcs]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
    psrc = os.path.join(CSRC, "peak_fp32.cu")
    if force or _stale(PEAK, [psrc]):
        subprocess.run([NVCC, *NVCC_FLAGS, "-o", PEAK, psrc], check=True)
    wsrc = os.path.join(CSRC, "synth_warp.c")
    if force or _stale(SYNTH, [wsrc]):
        subprocess.run([HOST_CC, "-O3", "-fPIC", "-fopenmp", "-shared", "-o", SYNTH, wsrc, "-lm"],
                       check=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
