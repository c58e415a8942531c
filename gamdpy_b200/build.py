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


def _includes(path, seen=None):
    """The file and every local header it includes, recursively."""
    seen = set() if seen is None else seen
    path = os.path.normpath(path)
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line.startswith("#include \""):
                _includes(os.path.join(os.path.dirname(path), line.split('"')[1]), seen)
    return seen


def build(verbose=False, force=False):
    """Compile the translation units whose sources or included headers are
    newer than their objects (all of them with force), then link."""
    objs, cmds = [], []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(CSRC, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, _includes(path)):
            cmds.append([NVCC, *ARCH, *FLAGS, "-c", path, "-o", obj])
    if not cmds and not _stale(LIB, objs):
        return LIB
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
