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
SOURCES = ["abi.cu", "grid.cu", "search.cu", "search_f32.cu", "search_f16.cu", "search_bf16.cu", "pipeline.cu",
           "mlp.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-Xcompiler", "-fPIC",
         "-I", str(ROOT / "include")]
LINK = ["-shared", "-cudart", "shared"]


def _digest():
    h = hashlib.sha1()
    for f in SOURCES + ["common.cuh", "search_impl.cuh"]:
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
    objdir = ROOT / "_build"
    objdir.mkdir(exist_ok=True)
    objs = [objdir / (Path(s).stem + ".o") for s in SOURCES]
    procs = []
    for s, o in zip(SOURCES, objs):       # one nvcc per translation unit, in parallel
        cmd = [NVCC] + FLAGS + ["-c", str(HERE / s), "-o", str(o)]
        if verbose:
            print(" ".join(cmd))
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    for s, pr in procs:
        _, err = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError(f"nvcc failed on {s}:\n{err[-6000:]}")
    r = subprocess.run([NVCC] + LINK + [str(o) for o in objs] + ["-o", str(tmp)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stderr[-6000:]}")
    os.replace(tmp, LIB)
    stamp.write_text(dg)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
