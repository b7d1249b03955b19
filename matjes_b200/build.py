"""Build the CUDA library in-tree for sm_100a (``python matjes_b200/build.py``).

Every translation unit is compiled to an object in parallel (the tiled kernels
are one unit per lattice shape), then linked into libmatjes_b200.so.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmatjes_b200.so")
OBJDIR = os.path.join(os.path.dirname(HERE), "_build", "obj")
SOURCES = ["mj_kernels.cu", "mj_tiled.cu", "mj_tiled_square_nn.cu", "mj_tiled_square2.cu", "mj_tiled_tri_nn.cu",
           "mj_tiled_tri3.cu", "mj_dipolar.cu", "mj_batch.cu", "mj_adjoint.cu", "mj_minimize.cu", "mj_mc.cu",
           "mj_gneb.cu", "mj_lattice.cpp", "mj_abi.cpp"]
HEADERS = ["mj_internal.hpp", "mj_device.cuh", "mj_shapes.hpp", "mj_tiled_impl.cuh", "mj_stencil.cuh",
           "mj_gneb.cuh", "mj_mc.cuh", os.path.join("..", "..", "include", "matjes_gpu.h")]
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


def _compile(src: str):
    obj = os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")
    cmd = [_nvcc(), *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    return src, obj, res


def build(force: bool = False, verbose: bool = False, jobs: int = 0) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(OBJDIR, exist_ok=True)
    jobs = jobs or max(1, min(len(SOURCES), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        results = list(ex.map(_compile, SOURCES))
    report = []
    for src, obj, res in results:
        report.append(f"=== {src}\n{res.stderr}")
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError(f"nvcc failed on {src}")
    tmp = OUT + ".tmp"
    link = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp,
            *[obj for _, obj, _ in results], "-lcufft"]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("link of libmatjes_b200.so failed")
    os.replace(tmp, OUT)
    text = "\n".join(report)
    if verbose:
        sys.stderr.write(text)
    with open(os.path.join(os.path.dirname(OBJDIR), "ptxas_report.txt"), "w") as f:
        f.write(text)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
