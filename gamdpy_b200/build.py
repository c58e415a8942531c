"""Build libgamdb200.so (sm_100a) in-tree with nvcc.

    python -m gamdpy_b200.build

The library is written next to this file; ``gamdpy_b200._lib`` loads it from
there and raises if it is missing.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgamdb200.so")
SOURCES = ["md_core.cu", "md_inst_nt1.cu", "md_inst_nt2.cu", "md_inst_ntg.cu", "md_cluster.cu", "analysis.cu",
           "adjoint.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "--expt-relaxed-constexpr"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    deps = [os.path.join(CSRC, s) for s in SOURCES] + [
        os.path.join(CSRC, h) for h in ("gdb_internal.cuh", "md_phases.cuh", "md_kernels.cuh", "md_cluster.cuh", "md_bricks.cuh")
    ] + [os.path.join(HERE, "..", "include", "gamdb200.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    objs, cmds = [], []
    for src in SOURCES:
        obj = os.path.join(CSRC, src.replace(".cu", ".o"))
        cmds.append([NVCC, *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    # translation units compile in parallel
    procs = []
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd))
        procs.append(subprocess.Popen(cmd))
    if any(p.wait() != 0 for p in procs):
        raise RuntimeError("nvcc failed")
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
