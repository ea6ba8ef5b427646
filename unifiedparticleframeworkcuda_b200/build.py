"""Build the in-tree CUDA libraries for sm_100a: libupf.so (the C ABI of
include/upf.h) and libupf_compat.so (the reference's own entry points of
include/upf_compat.h, over libupf.so).

    python -m unifiedparticleframeworkcuda_b200.build [--force] [--ptxas-v]

The library is compiled with -fmad=false: no float multiply-add contraction,
so every float operation rounds on its own like the reference's x86 CPU
build (the parity target). Host math (lookup tables, defaults) is compiled
with -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libupf.so")
COMPAT_LIB = os.path.join(HERE, "libupf_compat.so")
INCLUDE = os.path.abspath(os.path.join(HERE, "..", "include"))

CU_SOURCES = ["upf_sort.cu", "upf_pipeline.cu", "upf_rigid.cu", "upf_api.cu", "upf_batch.cu", "upf_adjoint.cu", "upf_noalloc.cu", "upf_scene.cu"]
CPP_SOURCES = ["upf_params.cpp", "upf_io.cpp"]
HEADERS = ["upf_common.cuh", "upf_internal.h", "upf_sys.h", "upf_tma.cuh"]
COMPAT_SOURCES = ["upf_compat.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def _deps():
    srcs = [os.path.join(CSRC, f) for f in CU_SOURCES + CPP_SOURCES + HEADERS]
    srcs += [os.path.join(CSRC, f) for f in COMPAT_SOURCES]
    srcs.append(os.path.join(INCLUDE, "upf.h"))
    srcs.append(os.path.join(INCLUDE, "upf_compat.h"))
    srcs.append(os.path.abspath(__file__))
    return srcs


def up_to_date() -> bool:
    newest = _newest(_deps())
    return all(os.path.exists(f) and os.path.getmtime(f) >= newest for f in (LIB, COMPAT_LIB))


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = True) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    common = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-I" + INCLUDE, "-I" + CSRC,
              "-Xcompiler", "-fPIC,-ffp-contract=off", "-ccbin", _cxx()] + ARCH
    if ptxas_verbose:
        common += ["-Xptxas", "-v"]
    jobs = []
    objs = []
    for f in CU_SOURCES:
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        jobs.append([nvcc, "-c", os.path.join(CSRC, f), "-o", obj] + common)
    for f in CPP_SOURCES:
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        jobs.append([_cxx(), "-c", os.path.join(CSRC, f), "-o", obj, "-O2", "-std=c++17", "-fPIC", "-pthread",
                     "-ffp-contract=off", "-Wall", "-I" + INCLUDE, "-I" + CSRC, "-I/usr/local/cuda/include"])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        for cmd, r in ex.map(run, jobs):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError("compile failed: " + " ".join(cmd[:3]))
            if ptxas_verbose or not quiet:
                sys.stderr.write(r.stderr)
    tmp = LIB + ".tmp"
    link = [nvcc, "-shared", "-o", tmp] + objs + ARCH + ["-Xcompiler", "-fPIC,-pthread", "-ccbin", _cxx()]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    # the compatibility layer: its own objects, linked against libupf.so and
    # finding it beside itself at run time
    cobjs = []
    for f in COMPAT_SOURCES:
        obj = os.path.join(BUILD, f + ".o")
        cobjs.append(obj)
        r = subprocess.run([nvcc, "-c", os.path.join(CSRC, f), "-o", obj] + common, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("compile failed: " + f)
    tmp = COMPAT_LIB + ".tmp"
    link = [nvcc, "-shared", "-o", tmp] + cobjs + ARCH + ["-L" + HERE, "-lupf", "-Xlinker", "-rpath,$ORIGIN",
                                                          "-Xcompiler", "-fPIC,-pthread", "-ccbin", _cxx()]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed: libupf_compat.so")
    os.replace(tmp, COMPAT_LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_verbose=a.ptxas_v, quiet=False))


if __name__ == "__main__":
    main()
