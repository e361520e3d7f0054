"""Build libnnsph.so (FP32, the product) and libnnsph64.so (the same source with
real = double, the FP64 run the FP32 path's error is stated against) in-tree for
sm_100a with nvcc (no JIT cache, no torch extension)."""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "nnsph.cu")
OUT = os.path.join(HERE, "libnnsph.so")
OUT64 = os.path.join(HERE, "libnnsph64.so")
DEPS = [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))] + [
    os.path.join(HERE, "..", "include", "nnsph.h")]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-shared",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def needs_build(out: str = OUT) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in DEPS if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Both libraries (compiled in parallel); returns the FP32 one's path."""
    jobs = []
    for out, extra in ((OUT, []), (OUT64, ["-DNN_FP64"])):
        if force or needs_build(out):
            cmd = [nvcc(), *NVCC_FLAGS, *extra, "-o", out + ".tmp", SRC]
            jobs.append((out, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    for out, p in jobs:
        so, se = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed for {os.path.basename(out)}:\n{so}\n{se}")
        if verbose:
            print(so, se)
        os.replace(out + ".tmp", out)
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose=True))
