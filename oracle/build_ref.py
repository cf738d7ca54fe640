"""Recipe: compile the reference's own CPU build of the hot path into ``oracle/_ref/``.

The reference keeps its kernels as C++ text inside Python modules and builds its CPU twin from that text
(``src/adock/cpukernel.py:81-142`` ``host_source``: compat header + ``mckernel._SRC`` + ``grid._KERNEL_SRC`` +
OpenMP launchers). This recipe imports those modules from a reference checkout (with empty stand-ins for
``cupy`` and ``rdkit``, which the text generation does not use), asks ``host_source`` for the text, and
compiles it with g++ into ``oracle/_ref/adock_ref_<AM>_<KM>.so``. The fitted grid kernel
(``src/adock/fit/gridfit.py:12-59``) has no CPU build in the reference; it is compiled the same way (the
reference's compat header + the kernel text) with a small OpenMP launcher written here.

Flags: the reference uses ``-O3 -march=native -ffast-math -fopenmp``; ``-march=native`` is replaced by
``-march=x86-64-v3`` because the built library travels to other hosts.

Outputs only into ``oracle/_ref/``. Test infrastructure: nothing in the product imports this.
Usage: ``python oracle/build_ref.py [--reference DIR]``. Without the argument the checkout is ``$ADOCK_REFERENCE``,
else the read-only mount of the build container (``CONTAINER_MOUNT``); ``locate_reference`` resolves it.
"""
import argparse
import os
import subprocess
import sys
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
CONTAINER_MOUNT = Path("/root/reference")   # where the build container mounts the reference checkout


def locate_reference(arg=None):
    """The reference checkout to build from (argument, then $ADOCK_REFERENCE, then the container mount), or None
    when none of them holds one."""
    for cand in (arg, os.environ.get("ADOCK_REFERENCE"), CONTAINER_MOUNT):
        if cand and (Path(cand) / "src" / "adock" / "cpukernel.py").exists():
            return Path(cand)
    return None
BUCKETS = [(64, 8), (64, 16), (64, 24), (96, 8), (96, 16), (96, 24)]
CXXFLAGS = ["-O3", "-march=x86-64-v3", "-ffast-math", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-std=c++17", "-w"]

FIT_LAUNCHER = r"""
extern "C" void launch_build_grid_fit(
    const float* rxyz, const int* rtype, const int n_rec, const float* rad_rec, const float* rad_lig, const int n_lt,
    const float* W, const float ox, const float oy, const float oz, const float spacing,
    const int nx, const int ny, const int nz, const float* prm, float* out)
{
    const long long npts = (long long)nx * ny * nz;
    #pragma omp parallel for schedule(dynamic, 256)
    for (long long p = 0; p < npts; ++p) {
        blockIdx.x = p;
        build_grid_fit(rxyz, rtype, n_rec, rad_rec, rad_lig, n_lt, W, ox, oy, oz, spacing, nx, ny, nz, prm, out);
    }
}
extern "C" void set_threads(int n) { omp_set_num_threads(n); }
"""


def _import_reference(ref: Path):
    for name in ("cupy", "rdkit", "rdkit.Chem"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.path.insert(0, str(ref / "src"))
    from adock import cpukernel  # noqa: E402
    from adock.fit import gridfit  # noqa: E402
    return cpukernel, gridfit


def _compile(src: str, so: Path):
    cpp = so.with_suffix(".cpp")
    cpp.write_text(src)
    tmp = so.with_name(so.name + f".{os.getpid()}.tmp")
    r = subprocess.run(["g++"] + CXXFLAGS + [str(cpp), "-o", str(tmp)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed for {so.name}:\n{r.stderr[-3000:]}")
    os.replace(tmp, so)
    cpp.unlink()          # keep only the built library: the generated text is the reference's source


def build(ref: Path, force: bool = False) -> list:
    if not (ref / "src" / "adock" / "cpukernel.py").exists():
        raise FileNotFoundError(f"no reference checkout at {ref}")
    OUT.mkdir(exist_ok=True)
    cpukernel, gridfit = _import_reference(ref)
    built = []
    for am, km in BUCKETS:
        so = OUT / f"adock_ref_{am}_{km}.so"
        if force or not so.exists():
            src, _ = cpukernel.host_source(am, km)
            _compile(src, so)
        built.append(so)
    so = OUT / "adock_ref_gridfit.so"
    if force or not so.exists():
        _compile(cpukernel._COMPAT + gridfit._SRC + FIT_LAUNCHER, so)
    built.append(so)
    return built


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    ref = locate_reference(a.reference)
    if ref is None:
        ap.error("no reference checkout: give --reference DIR or set ADOCK_REFERENCE")
    for p in build(ref, a.force):
        print(p)
