"""Build recipe of the reference harness: compiles oracle/ref_harness.cu against the reference's
own headers, where they lie, into oracle/_ref/libawref.so (nvcc, sm_100a).  Test infrastructure."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUT_DIR, "libawref.so")
SRC = os.path.join(HERE, "ref_harness.cu")


def build(ref_root: str, force: bool = False) -> str | None:
    inc = os.path.join(ref_root, "include")
    if not os.path.isdir(inc):
        return None
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [os.environ.get("NVCC", "nvcc"), "-std=c++20", "--expt-relaxed-constexpr", "-rdc=true",
           "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-shared", "-Xcompiler", "-fPIC",
           "-w", "-I", inc, SRC, "-o", OUT]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("reference harness build failed")
    return OUT


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else "/root/reference", force=True))
