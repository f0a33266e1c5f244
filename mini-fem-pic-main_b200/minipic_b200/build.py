"""Builds lib/libminipic_cuda.so for sm_100a with nvcc (no JIT cache: the
library is built in-tree so it ships with the repository)."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libminipic_cuda.so")
INCLUDE = os.path.join(REPO, "include")

CU_SOURCES = ["mp_api.cu", "mp_push.cu", "mp_field.cu", "mp_solve.cu", "mp_noalloc.cu", "mp_adjoint.cu", "mp_inject.cu", "mp_sparse.cu", "mp_mesh.cu"]
CPP_SOURCES = ["mp_host.cpp", "mp_output.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "minipic_cuda.h")]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest(deps):
        return LIB
    nvcc = _nvcc()
    common = ["-O3", "-std=c++17", "-I" + INCLUDE, "-I" + CSRC, "-Xcompiler", "-fPIC"]
    objs = []
    cmds = []
    for src in CU_SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmds.append([nvcc, *ARCH, "-lineinfo", *common, "-Xptxas", "-warn-spills", "-c",
                     os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    for src in CPP_SOURCES:
        obj = os.path.join(objdir, src + ".o")
        # host setup arithmetic must not be contracted into FMAs (bit-exact geometry)
        cmds.append(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
                     "-I" + INCLUDE, "-I" + CSRC, "-I/usr/local/cuda/include", "-c",
                     os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    procs = []
    for c in cmds:
        if verbose:
            print(" ".join(c))
        procs.append((c, subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for c, p in procs:
        out, _ = p.communicate()
        if out and (verbose or p.returncode):
            sys.stdout.write(out)
        if p.returncode:
            failed.append(c[-3] if c[0] == "g++" else c[-3])
    if failed:
        raise RuntimeError(f"compilation failed: {failed}")
    link = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-cudart=static"]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
