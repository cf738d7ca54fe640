"""Build the oracle's C restatement (oracle/port.c) into oracle/liboracle_port.so (gcc, OpenMP).

Test infrastructure only. Usage: ``python oracle/build_port.py``."""
import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "port.c"
LIB = HERE / "liboracle_port.so"
CFLAGS = ["-O2", "-std=c11", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off"]


def build(force=False):
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    tmp = LIB.with_name(LIB.name + f".{os.getpid()}.tmp")
    r = subprocess.run(["gcc"] + CFLAGS + [str(SRC), "-o", str(tmp), "-lm"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"gcc failed:\n{r.stderr[-4000:]}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
