"""Build the sm_100a library and its Python module in-tree.

    python chemtoolscuda_b200/build.py          # incremental
    python chemtoolscuda_b200/build.py --clean

Produces
  chemtoolscuda_b200/libchemtools_cuda.so          the C ABI (include/chemtools_cuda.h)
  chemtoolscuda_b200/_chemtools_cuda<EXT_SUFFIX>   the pybind11 module (Molecule)
Objects go to chemtoolscuda_b200/_build/.  Every CUDA translation unit is
compiled for sm_100a only (-gencode arch=compute_100a,code=sm_100a).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libchemtools_cuda.so")
EXT = os.path.join(HERE, "_chemtools_cuda" + sysconfig.get_config_var("EXT_SUFFIX"))

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-pthread",
              "--expt-relaxed-constexpr", "-I" + INCLUDE] + ARCH
CU_SOURCES = ["ctc_basis.cu", "ctc_ao.cu", "ctc_local.cu", "ctc_tc.cu", "ctc_esp.cu",
              "ctc_adjoint.cu", "ctc_api.cu", "ctc_noalloc.cu", "ctc_fchk.cpp",
              "ctc_molden.cpp", "ctc_wfn.cpp"]
HEADERS = ["ctc_internal.h", "ctc_terms.inc", "ctc_ao_poly.inc", "ctc_tiles.cuh", "ctc_split.cuh",
           "ctc_finalize.cuh",
           "ctc_wfnfile.h"]


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "chemtools_cuda.h")]
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, os.path.splitext(s)[0] + ".o")
        objs.append(obj)
        if _newer([src] + hdrs, obj):
            jobs.append([NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for r in ex.map(_run, jobs):
                if verbose and r.stderr:
                    print(r.stderr)
    if _newer(objs, LIB):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs +
             ["-Xcompiler", "-pthread", "-lcudart"])
    # pybind11 module, linked against the library with an $ORIGIN rpath
    import pybind11
    pysrc = os.path.join(CSRC, "pymodule.cpp")
    if _newer([pysrc, LIB, os.path.join(INCLUDE, "chemtools_cuda.h")], EXT):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", pysrc, "-o", EXT,
              "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"],
              "-I" + os.path.join(CUDA_HOME, "include"), "-I" + INCLUDE,
              "-L" + HERE, "-lchemtools_cuda", "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart",
              "-Wl,-rpath,$ORIGIN"])
    return LIB


def clean():
    shutil.rmtree(BUILD, ignore_errors=True)
    for f in (LIB, EXT):
        if os.path.exists(f):
            os.remove(f)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    if a.clean:
        clean()
    print(build(verbose=a.v))
    sys.exit(0)
