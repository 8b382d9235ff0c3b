"""Build the in-tree C-ABI library ``ebsdtorch_b200/_lib/libebsd_b200.so``.

Every ``csrc/*.cu`` file is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) and linked into one shared
library with the static CUDA runtime. Usage: ``python -m ebsdtorch_b200.build``.
Objects are rebuilt only when a source or header is newer than the library.
``--check`` builds ``_lib/libebsd_b200_check.so`` with -DEBSD_CHECK (device
checks of computed offsets that record a failing line instead of accessing
memory; loaded when EBSD_CHECK_BUILD=1).
"""

from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libebsd_b200.so")
LIB_CHECK = os.path.join(LIBDIR, "libebsd_b200_check.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]
# per-file extra flags: the FP64 grid must round like the CPU oracle
FILE_FLAGS = {"grid.cu": ["-fmad=false"]}


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build ebsdtorch_b200")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _newest_input() -> float:
    files = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return max(os.path.getmtime(f) for f in files)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False, check: bool = False) -> str:
    lib = LIB_CHECK if check else LIB
    if not force and os.path.exists(lib) and os.path.getmtime(lib) >= _newest_input():
        return lib
    nvcc = _nvcc()
    objdir = os.path.join(LIBDIR, "obj_check" if check else "obj")
    os.makedirs(objdir, exist_ok=True)
    extra = (["-Xptxas", "-v"] if ptxas_info else []) + (["-DEBSD_CHECK"] if check else [])

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc, *ARCH, *FLAGS, *FILE_FLAGS.get(os.path.basename(src), []), *extra, "-I", INCLUDE, "-c", src,
               "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{r.stderr}")
        return obj, r.stderr

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, sources()))
    if verbose or ptxas_info:
        for _, err in results:
            if err.strip():
                print(err, file=sys.stderr)
    objs = [o for o, _ in results]
    tmp = lib + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force, verbose=True, ptxas_info="--ptxas-info" in sys.argv, check="--check" in sys.argv))
