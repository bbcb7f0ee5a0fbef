"""Build libdec_b200.so (sm_100a) in-tree with nvcc.

    python combinatorialspaces.jl_b200/build.py [--force]

Objects go to ``_build/``, the library to ``_lib/libdec_b200.so``.  The geometry, wedge and
operator translation units are compiled with ``-fmad=false`` so their FP64 arithmetic follows
the reference's operation order exactly; the multigrid kernels keep FMA contraction.
"""
import concurrent.futures
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "_lib" / "libdec_b200.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", f"-I{INCLUDE}", f"-I{CSRC}",
          "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
EXACT = {"mesh.cu", "wedge.cu", "ops.cu"}   # no FMA contraction
SOURCES = ["mesh.cu", "wedge.cu", "ops.cu", "mg.cu", "mlp.cu", "tune.cpp", "capi.cpp"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not pathlib.Path(exe).exists():
        raise RuntimeError("nvcc not found")
    return exe


def _compile(src: str, force: bool) -> pathlib.Path:
    s = CSRC / src
    o = BUILD / (src + ".o")
    deps = [s] + list(CSRC.glob("*.cuh")) + [INCLUDE / "dec_b200.h"]
    if not force and o.exists() and all(o.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return o
    flags = list(COMMON)
    if src.endswith(".cu"):
        flags += ARCH
        if src in EXACT:
            flags += ["-fmad=false"]
    cmd = [nvcc(), *flags, "-c", str(s), "-o", str(o)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if "spill" in r.stderr and "0 bytes spill" not in r.stderr:
        sys.stderr.write(r.stderr)
    return o


def build(force: bool = False) -> pathlib.Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), SOURCES))
    if force or not LIB.exists() or any(LIB.stat().st_mtime < o.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
