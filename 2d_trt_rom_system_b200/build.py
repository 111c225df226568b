"""Builds libtrt_sweep.so (the CUDA library behind include/trt_sweep.h) in place, for sm_100a.

The library is compiled with --fmad=false: every multiply-add that should fuse is written as an
explicit fma in the source, and every other operation rounds once, as in the reference Fortran.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libtrt_sweep.so")
SOURCES = ["trt_api.cu", "mgqd.cu", "rom.cu"]
HEADERS = ["aux_kernels.cuh", "dropin_kernels.cuh", "gqd_kernels.cuh", "handle_hooks.h", "layout.cuh", "mgqd_kernels.cuh",
           "ptx.cuh", "scb_cell.h",
           "sweep_kernel.cuh", "tstep_kernels.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIBS = ["-lcusolver", "-lcublas"]   # the SVD / eigenpairs / products of POD and DMD (rom.cu)
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC", "-diag-suppress", "177"]
OBJDIR = os.path.join(HERE, "_build")


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "trt_sweep.h"),
                                                                 os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compile the library if a source is newer than it: the translation units in parallel, then one
    link.  Returns the path of the .so."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OBJDIR, exist_ok=True)
    objs = [os.path.join(OBJDIR, os.path.splitext(s)[0] + ".o") for s in SOURCES]
    cmds = [[_nvcc()] + NVCC_FLAGS + ARCH + ["-I" + INCLUDE, "-I" + CSRC, "-c", "-o", o, os.path.join(CSRC, s)]
            for s, o in zip(SOURCES, objs)]
    if verbose:
        for c in cmds:
            print(" ".join(c), file=sys.stderr)
    with ThreadPoolExecutor(len(cmds)) as ex:
        procs = list(ex.map(lambda c: subprocess.run(c), cmds))
    if any(p.returncode for p in procs):
        raise subprocess.CalledProcessError(1, "nvcc")
    link = [_nvcc(), "-shared"] + ARCH + ["-o", LIB + ".tmp"] + objs + LIBS
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
