"""Build recipe of the reference harness: compiles oracle/ref_harness.cu against the reference's
own headers, where they lie, into oracle/_ref/libawref.so (nvcc, sm_100a).  Test infrastructure.

The reference tree is found at $AW_REFERENCE_ROOT, else at DEFAULT_REFERENCE_ROOT.

The harness links its own static CUDA runtime.  Everything but the harness's entry points is hidden
and the library binds its own symbols first (-Bsymbolic): a process that has already loaded another
CUDA runtime globally (torch loads libcudart with RTLD_GLOBAL) must not interpose its runtime
functions on the harness's kernel registration and launches.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUT_DIR, "libawref.so")
SRC = os.path.join(HERE, "ref_harness.cu")
DEFAULT_REFERENCE_ROOT = "/root/reference"


def reference_root() -> str:
    return os.environ.get("AW_REFERENCE_ROOT", DEFAULT_REFERENCE_ROOT)


def build(ref_root: str | None = None, force: bool = False) -> str | None:
    inc = os.path.join(ref_root or reference_root(), "include")
    if not os.path.isdir(inc):
        return None
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(SRC),
                                                                           os.path.getmtime(__file__)):
        return OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [os.environ.get("NVCC", "nvcc"), "-std=c++20", "--expt-relaxed-constexpr", "-rdc=true",
           "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-shared",
           "-Xcompiler", "-fPIC,-fvisibility=hidden", "-Xlinker", "-Bsymbolic",
           "-w", "-I", inc, SRC, "-o", OUT]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("reference harness build failed")
    return OUT


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else None, force=True))
