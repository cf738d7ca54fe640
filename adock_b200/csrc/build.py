"""Build ``libadock_b200.so`` (sm_100a) in-tree with nvcc.

Usage: ``python -m adock_b200.csrc.build [--force]``. The library lands next to the package
(``adock_b200/libadock_b200.so``) so that it travels with the source tree."""
import hashlib
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
ROOT = PKG.parent
LIB = PKG / "libadock_b200.so"
SOURCES = ["abi.cu", "grid.cu", "search.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-Xcompiler", "-fPIC",
         "-shared", "-cudart", "shared", "-I", str(ROOT / "include")]


def _digest():
    h = hashlib.sha1()
    for f in SOURCES + ["common.cuh"]:
        h.update((HERE / f).read_bytes())
    h.update((ROOT / "include" / "adock_b200.h").read_bytes())
    h.update(" ".join(FLAGS).encode())
    return h.hexdigest()


def build(force=False, verbose=False):
    stamp = LIB.with_suffix(".so.sha1")
    dg = _digest()
    if not force and LIB.exists() and stamp.exists() and stamp.read_text() == dg:
        return LIB
    tmp = LIB.with_name(LIB.name + f".{os.getpid()}.tmp")
    cmd = [NVCC] + FLAGS + [str(HERE / s) for s in SOURCES] + ["-o", str(tmp)]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{r.stderr[-6000:]}")
    os.replace(tmp, LIB)
    stamp.write_text(dg)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
