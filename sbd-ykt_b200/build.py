"""Build the sbdx CUDA library (sm_100a) and the C++ drop-in sample in place.

    python sbd-ykt_b200/build.py          # libsbdx.so (+ the diag sample binary)

The shared library is written next to this file so that it travels with the
repository snapshot; nothing is installed.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libsbdx.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_lib(force: bool = False) -> str:
    """Compiles every csrc/*.cu to an object (in parallel, under _build/) and
    links libsbdx.so; sources whose object is newer than them and than the
    shared headers are not recompiled."""
    srcs = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
    hdrs = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + [os.path.join(ROOT, "include", "sbdx.h")]
    if not force and not _stale(LIB, srcs + hdrs):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", host_cxx(),
             "-I" + os.path.join(ROOT, "include")]
    objs, jobs = [], []
    for src in srcs:
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            jobs.append([nvcc(), *flags, "-c", "-o", obj, src])
    procs = [subprocess.Popen(cmd) for cmd in jobs]
    failed = [cmd[-1] for cmd, p in zip(jobs, procs) if p.wait() != 0]
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(os.path.basename(f) for f in failed))
    subprocess.run([nvcc(), *ARCH, "-shared", "-ccbin", host_cxx(), "-o", LIB, *objs], check=True)
    return LIB


def build_sample(force: bool = False) -> str | None:
    """The C++ drop-in sample driver (cpp/diag_main.cc) over the header API."""
    src = os.path.join(HERE, "cpp", "diag_main.cc")
    if not os.path.exists(src):
        return None
    out = os.path.join(HERE, "cpp", "sbd_diag")
    deps = [src, LIB] + sorted(glob.glob(os.path.join(HERE, "cpp", "include", "sbd", "*.h")))
    if not force and not _stale(out, deps):
        return out
    cmd = [host_cxx(), "-std=c++17", "-O2", "-I" + os.path.join(HERE, "cpp", "include"),
           "-I" + os.path.join(ROOT, "include"), "-o", out, src, "-L" + HERE, "-lsbdx",
           "-Wl,-rpath,$ORIGIN/..", "-L/usr/local/cuda/lib64", "-lcudart"]
    subprocess.run(cmd, check=True)
    return out


def main(argv=None):
    force = "--force" in (argv or sys.argv[1:])
    print(build_lib(force))
    s = build_sample(force)
    if s:
        print(s)


if __name__ == "__main__":
    main()
