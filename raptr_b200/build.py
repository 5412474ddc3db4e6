"""Builds the in-tree CUDA library raptr_b200/libraptr_b200.so for sm_100a.

    python -m raptr_b200.build

Every translation unit is compiled with nvcc for sm_100a only; host code is
compiled without floating-point contraction, and the system-matrix unit also
with -fmad=false (its exact paths use explicit round-to-nearest intrinsics).
"""
from __future__ import annotations

import os
import subprocess
from concurrent.futures import ThreadPoolExecutor
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libraptr_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off",
          "-ccbin", "/usr/bin/g++"]
UNITS = {
    "api.cu": [],
    "kernels_sm.cu": ["-fmad=false"],
    "kernels_util.cu": [],
    "kernels_mlem.cu": [],
    "kernels_transpose.cu": [],
    "kernels_precision.cu": [],
    "kernels_batch.cu": [],
    "server.cu": [],
    "h5lite.cpp": [],
    "devmem.cu": [],
    "mlem_noalloc.cu": [],
}


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, extra=()) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "raptr_b200.h"))
    headers.append(os.path.join(HERE, "..", "include", "raptr_b200_h5.h"))
    objs, jobs = [], []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OBJ, os.path.splitext(unit)[0] + ".o")
        objs.append(obj)
        if _stale(obj, [src, __file__] + headers):
            jobs.append((unit, [_nvcc(), "-c", src, "-o", obj] + ARCH + COMMON + flags + list(extra)))

    def compile_unit(job):
        unit, cmd = job
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {unit}:\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr)

    # the translation units compile independently
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        list(pool.map(compile_unit, jobs))
    if _stale(LIB, objs):
        cmd = [_nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-ccbin", "/usr/bin/g++"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_drivers(headers)
    return LIB


DRIVERS = ("reco", "backprojection", "pureSMCalculation")
BIN = os.path.join(HERE, "bin")


def build_drivers(headers=()) -> list:
    """The command-line drivers (reference argv), host C++ over the
    library: raptr_b200/bin/{reco,backprojection,pureSMCalculation}."""
    os.makedirs(BIN, exist_ok=True)
    src_dir = os.path.join(HERE, "drivers")
    inc = os.path.join(HERE, "..", "include")
    cuda = os.path.dirname(os.path.dirname(os.path.realpath(_nvcc()))) if os.path.sep in _nvcc() else "/usr/local/cuda"
    out = []
    for d in DRIVERS:
        src = os.path.join(src_dir, d + ".cpp")
        exe = os.path.join(BIN, d)
        out.append(exe)
        deps = [src, os.path.join(src_dir, "common.hpp"), LIB, os.path.join(inc, "raptr_b200.hpp")] + list(headers)
        if _stale(exe, deps):
            cmd = ["/usr/bin/g++", "-std=c++17", "-O2", src, "-o", exe, f"-I{inc}", f"-I{cuda}/include", f"-L{HERE}",
                   "-lraptr_b200", f"-Wl,-rpath,{HERE}", f"-L{cuda}/lib64", "-lcudart", f"-Wl,-rpath,{cuda}/lib64"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"driver {d} failed to build:\n{r.stderr}")
    return out


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(verbose=v, extra=extra))
