"""Build recipe of the sm_100a library (nvcc -> libanitowave.so, in-tree)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
SOURCES = ["aw_grid.cu", "aw_particles.cu", "aw_solver.cu", "aw_flip.cu", "aw_adjoint.cu", "aw_noalloc.cu",
           "aw_output.cu"]
OUT = os.path.join(PKG, "libanitowave.so")
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-fvisibility=hidden",
    "--expt-relaxed-constexpr", "-Xptxas", "-v",
]


def sources():
    return [os.path.join(HERE, s) for s in SOURCES]


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = sources() + [os.path.join(HERE, "aw_internal.cuh"), os.path.join(ROOT, "include", "anitowave.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    cmd = [NVCC, *FLAGS, "-I", os.path.join(ROOT, "include"), "-I", HERE, *sources(), "-o", OUT]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed")
    # register / spill / shared-memory report of every kernel, kept out of the tracked tree
    os.makedirs(os.path.join(PKG, "_build"), exist_ok=True)
    with open(os.path.join(PKG, "_build", "ptxas_info.txt"), "w") as f:
        f.write(res.stderr.replace(ROOT + os.sep, ""))  # paths relative to the repository
    if verbose:
        sys.stderr.write(res.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
