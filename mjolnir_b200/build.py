"""Builds the sm_100a shared library of the package in place.

``python -m mjolnir_b200.build`` (or ``build()``) compiles every CUDA and C++
source under ``csrc/`` with nvcc into ``mjolnir_b200/libmjolnir_b200.so``.
The library is rebuilt only when a source is newer than it.
"""
from __future__ import annotations

import concurrent.futures
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libmjolnir_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "-Xcompiler", "-fvisibility=hidden"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) \
        + glob.glob(os.path.join(INCLUDE, "*.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and not _stale():
        return LIB
    build_dir = os.path.join(HERE, "_build")
    os.makedirs(build_dir, exist_ok=True)
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    objs = []
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) \
        + glob.glob(os.path.join(INCLUDE, "*.h"))
    newest_header = max((os.path.getmtime(h) for h in headers), default=0.0)
    cmds = []
    for src in sources():
        obj = os.path.join(build_dir, os.path.basename(src) + ".o")
        objs.append(obj)
        # an object is recompiled when its source or any header is newer
        if not force and not ptxas_info and os.path.exists(obj) and \
                os.path.getmtime(obj) >= max(os.path.getmtime(src), newest_header):
            continue
        cmds.append([nvcc(), *ARCH, *NVFLAGS, *extra, "-I", INCLUDE, "-c", src, "-o", obj])
    # the translation units compile side by side (the pair kernels' unit
    # alone takes minutes)
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
        for f in [ex.submit(subprocess.run, cmd, check=True, env=env) for cmd in cmds]:
            f.result()
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    subprocess.run(cmd, check=True, env=env)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
