"""Build the CUDA library in-tree for sm_100a (``python -m matjes_b200.build``)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmatjes_b200.so")
SOURCES = ["mj_kernels.cu", "mj_tiled.cu", "mj_dipolar.cu", "mj_lattice.cpp", "mj_abi.cpp"]
HEADERS = ["mj_internal.hpp", "mj_device.cuh", "mj_shapes.hpp", os.path.join("..", "..", "include", "matjes_gpu.h")]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3",
    "-Xptxas", "-v",
    "-diag-suppress", "177",
]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES] + [os.path.join(CSRC, h) for h in HEADERS]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in sources() if os.path.exists(s))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    tmp = OUT + ".tmp"
    cmd = [_nvcc(), *NVCC_FLAGS, "-shared", "-o", tmp, *[os.path.join(CSRC, s) for s in SOURCES], "-lcufft"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc build of libmatjes_b200.so failed")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(tmp, OUT)
    with open(os.path.join(HERE, "ptxas_report.txt"), "w") as f:
        f.write(res.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
