"""In-tree build of libmfcfd_b200.so (nvcc, sm_100a).

The shared library is written next to this file so it travels with the
source tree; ``python -m mfcfd_b200.build`` rebuilds it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libmfcfd_b200.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("primal_fp64.cu", "api.cu")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in ("primal.h", "lskum_device.cuh")] + [
    os.path.join(ROOT, "include", "mfcfd_b200.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: cannot build libmfcfd_b200.so")


def command(out: str = LIB, extra=()) -> list:
    # -ffp-contract=off: the host-side set-up (normals, split masks, limiter
    # epsilon) must round exactly like the reference's arithmetic.
    return [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-I", os.path.join(ROOT, "include"),
            "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared", *extra, "-o", out, *SOURCES]


def up_to_date(out: str = LIB) -> bool:
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(s) <= t for s in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    cmd = command()
    tmp = LIB + ".tmp"
    cmd[cmd.index(LIB)] = tmp
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose and res.stderr:
        print(res.stderr, file=sys.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
