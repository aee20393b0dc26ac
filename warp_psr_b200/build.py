"""Builds ``libpsr_b200.so`` in-tree for sm_100a with nvcc (no JIT, no torch extension).

``python -m warp_psr_b200.build`` compiles every ``csrc/*.cu`` in parallel into
``_build/*.o`` and links the shared library next to this file.  FMA contraction is off
(``--fmad=false`` on the device, ``-ffp-contract=off`` on the host) so every scalar
operation rounds where the reference's (``fuse_fp: False``) does.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "_build"
LIB = HERE / "libpsr_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
         "-Xptxas", "-warn-spills", "--expt-relaxed-constexpr"]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libpsr_b200")
    return path


def _compile(src, verbose):
    obj = OUT / (src.stem + ".o")
    deps = list(CSRC.glob("*.cuh")) + list((HERE.parent / "include").glob("*.h*")) + [src]
    if obj.exists() and obj.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return obj, ""
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stderr}")
    return obj, res.stderr if verbose else ""


def build(verbose=False):
    OUT.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    with ThreadPoolExecutor(max_workers=min(len(sources), os.cpu_count() or 4)) as pool:
        results = list(pool.map(lambda s: _compile(s, verbose), sources))
    objs = [r[0] for r in results]
    for _, log in results:
        if log:
            sys.stderr.write(log)
    if not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode:
            raise RuntimeError(f"link failed:\n{res.stderr}")
    return LIB


INCLUDE = HERE.parent / "include"


def build_user_library(sources, output, extra_flags=()):
    """Compiles CUDA sources of an application that evaluates reconstructed fields inside its
    own kernels (``#include "psr_field.cuh"``, then ``psr_evaluate_field(handle, x, y, z)``)
    into a shared library for sm_100a.  The application's own flags apply (FMA contraction
    stays on by default); the header's arithmetic does not depend on them.  Returns the path."""
    output = Path(output)
    cmd = [nvcc(), *ARCH, "-std=c++17", "-O3", "-lineinfo", "-I", str(INCLUDE), "-Xcompiler", "-fPIC", "-shared",
           *map(str, sources), "-o", str(output), *extra_flags]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode:
        raise RuntimeError(f"nvcc failed:\n{res.stderr}")
    return output


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
