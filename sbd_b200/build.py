"""Build the in-tree shared library sbd_b200/libsbdgpu.so (sm_100a) and the
sample driver sbd_b200/bin/diag.  Plain nvcc/g++ invocations, no JIT cache."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsbdgpu.so")
SOURCES = ["api.cu", "tables.cu", "sigma.cu", "misc.cu", "tc_ab.cu", "noalloc.cu", "stored.cu", "roots.cu", "batch.cu", "learned.cu", "gemm_same.cu", "genop.cu", "genop_fcidump.cu", "rdm.cu", "ozaki.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"), "nvcc"):
        if os.path.sep not in c or os.path.exists(c):
            return c
    return "nvcc"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(force: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, "internal.cuh"), os.path.join(ROOT, "include", "sbdgpu.h"),
                   os.path.join(HERE, "include", "sbd_gpu", "generalop.h"), os.path.join(HERE, "include", "sbd_gpu", "tpb.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", "g++",
               "-I", os.path.join(ROOT, "include"), "-I", os.path.join(HERE, "include"), "-c", s, "-o", o]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append(subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
        objs.append(o)
    failed = False
    for p in procs:
        out, _ = p.communicate()
        if out.strip():
            print(out, file=sys.stderr)
        failed |= p.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed")
    subprocess.run([nvcc(), *ARCH, "-shared", "-ccbin", "g++", "-o", LIB, *objs, "-lcudart", "-lcublas"], check=True)
    return LIB


DRIVER = os.path.join(HERE, "bin", "diag")


def build_driver(force: bool = False) -> str:
    """The sample driver (same flags as the reference sample) linked to libsbdgpu.so."""
    lib = build_lib()
    src = os.path.join(HERE, "samples", "diag.cc")
    hdr = os.path.join(HERE, "include", "sbd_gpu", "tpb.h")
    if not force and not _stale(DRIVER, [src, hdr, lib]):
        return DRIVER
    os.makedirs(os.path.dirname(DRIVER), exist_ok=True)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(HERE, "include"), "-I", os.path.join(ROOT, "include"),
                    src, "-o", DRIVER, "-L", HERE, "-lsbdgpu", "-Wl,-rpath,$ORIGIN/.."], check=True)
    return DRIVER


if __name__ == "__main__":
    build_lib(force="--force" in sys.argv, verbose="-v" in sys.argv)
    build_driver(force="--force" in sys.argv)
    print(LIB, DRIVER)
