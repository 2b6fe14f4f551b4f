"""Build the sm_100a shared library ``romspath_b200/_lib/libromspath_b200.so``.

The library is the C ABI of ``include/romspath_gpu.h``.  The kernel unit is
compiled with ``-fmad=false`` so that FP64 arithmetic rounds exactly like the
reference's evaluation order (no FMA contraction).  nvcc cross-compiles for
sm_100a without a GPU present.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from typing import List

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(OUT_DIR, "libromspath_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC]

# (source, extra flags)
UNITS = [
    ("rp_kernels.cu", ["-fmad=false"]),
    ("rp_noalloc.cu", ["-fmad=false"]),
    ("rp_mixed.cu", []),          # mixed-precision form: FMA contraction allowed
    ("rp_sort.cu", []),           # re-sorting of the particle state (no arithmetic on values)
    ("rp_adjoint.cu", ["-fmad=false"]),   # adjoint pair: double and dual instantiations agree
    ("rp_init.cu", ["-fmad=false"]),      # LL2ij on the device, nest maps on the host
    ("rp_api.cu", []),
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources() -> List[str]:
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(INCLUDE, "romspath_gpu.h"))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _sources())


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    nvcc = _nvcc()
    os.makedirs(OUT_DIR, exist_ok=True)
    objs, procs = [], []
    for src, extra in UNITS:          # the units compile in parallel
        obj = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
        cmd = [nvcc, *COMMON, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        objs.append(obj)
    for src, pr in procs:
        out, err = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{out}\n{err}")
        if ptxas_info or verbose:
            sys.stdout.write(err)
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv, force=True)
    print(LIB)
