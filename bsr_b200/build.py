"""Build bsr_b200/libbsrgpu.so (sm_100a) in-tree with nvcc.

The table kernels (rk_tables.cu) and the reference-order density/convol
kernels (convol.cu) are compiled with --fmad=false so they reproduce the
Fortran arithmetic exactly; the assembly and eigensolve units use FMA.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libbsrgpu.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "-I" + os.path.join(HERE, "..", "include")]
UNITS = {
    "capi.cu": [],
    "rk_tables.cu": ["--fmad=false"],
    "convol.cu": ["--fmad=false"],
    "assemble.cu": [],
    "diag_hd.cu": [],
    "noalloc.cu": [],
    "eigen.cu": [],
    "post.cu": [],
    "dgemm.cu": [],
    "refine.cu": [],
    "tridiag_dc.cu": [],
    "syevd2.cu": [],
    "tc_mixed.cu": [],
    "tc_ozaki.cu": [],
    "chan_eig.cu": [],
    "dense_chol.cu": [],
}


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    headers.append(os.path.join(HERE, "..", "include", "bsr_b200.h"))
    hdr_mtime = max(os.path.getmtime(h) for h in headers)
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime):
            continue
        cmd = [nvcc()] + ARCH + COMMON + extra + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    cmd = [nvcc()] + ARCH + ["-shared", "-o", OUT] + objs + [
        "-L/usr/local/cuda/lib64", "-lcublas", "-lcusolver", "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
