"""Builds the native parts of monalisa_b200 in-tree (no JIT cache):

* ``_lib/libmonalisa_gpu.so`` -- the CUDA library behind include/monalisa_gpu.h,
  compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
* ``_lib/libmexshim.so`` -- the project's MEX-API shim;
* ``_lib/mex/<name>.so`` -- the drop-in MEX gateways (reference names and
  argument layouts), linked against the shim and libmonalisa_gpu.so;
* ``driver/_bin/monalisa_driver`` -- the standalone C++ reconstruction driver
  (driver/monalisa_driver.cpp) on the C ABI.

Usage: ``python -m monalisa_b200.build`` (or ``build()`` from Python).
Object files go to ``_build/`` (git-ignored).  Rebuilds only what changed.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "_lib")
OBJ = os.path.join(ROOT, "_build", "obj")
INCLUDE = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
# The system g++ (the environment's CXX wrapper may lack the OpenMP runtime).
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "-ccbin", CXX] + ARCH

GATEWAYS = [
    "bmGridder_n2u_leight1_mex", "bmGridder_n2u_leight2_mex", "bmGridder_n2u_leight3_mex",
    "bmGridder_n2u_mex",
    "bmSparseMat_cC_oBlock_omp_mex", "bmSparseMat_cC_oBlock_mex", "bmSparseMat_cR_oBlock_mex",
    "bmSparseMat_rC_oBlock_mex", "bmSparseMat_rC_oBlock_omp_mex", "bmSparseMat_r_nJump2index_mex",
    "bmSparseMat_rR_oBlock_mex", "bmSparseMat_cR_nBlock_omp_mex", "bmSparseMat_rR_nBlock_omp_mex",
    "bmSparseMat_cC_oBlock_2_omp_mex",
    "bmShanna1_CUFFT_omp_mex", "bmShanna2_CUFFT_omp_mex", "bmShanna3_CUFFT_omp_mex",
    "bmNakatsha1_CUFFT_omp_mex", "bmNakatsha2_CUFFT_omp_mex", "bmNakatsha3_CUFFT_omp_mex",
    "bmIDF1_CUFFT_mex", "bmIDF2_CUFFT_mex", "bmIDF3_CUFFT_mex",
]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(os.path.join(LIB, "mex"), exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
    so = os.path.join(LIB, "libmonalisa_gpu.so")
    # a library newer than every source needs no objects (they need not be
    # present: only the library travels with the sources)
    lib_current = not _newer(so, cu + cpp + headers)
    objs, cmds = [], []
    for src in cu:
        o = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(o)
        if _newer(o, [src] + headers):
            cmds.append([NVCC, *NVCC_FLAGS, "-I", INCLUDE, "-c", src, "-o", o])
    for src in cpp:
        o = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(o)
        if _newer(o, [src] + headers):
            cmds.append([CXX, "-O3", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-I", INCLUDE,
                         "-I", os.path.join(CUDA_HOME, "include"), "-c", src, "-o", o])
    if lib_current:
        cmds = []
    with ThreadPoolExecutor(jobs or min(8, os.cpu_count() or 4)) as ex:
        list(ex.map(_run, cmds))
    if not lib_current and _newer(so, objs):
        _run([NVCC, *ARCH, "-shared", "-o", so, *objs, "-L", os.path.join(CUDA_HOME, "lib64"),
              "-lcufft", "-lcudart", "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")])
    shim_src = os.path.join(CSRC, "mexshim", "mexshim.cpp")
    shim = os.path.join(LIB, "libmexshim.so")
    if _newer(shim, [shim_src, os.path.join(CSRC, "mexshim", "mex.h")]):
        _run([CXX, "-O2", "-fPIC", "-shared", "-std=c++17", "-I", os.path.join(CSRC, "mexshim"),
              "-o", shim, shim_src])
    gw_src = os.path.join(CSRC, "mex", "gateways.cpp")
    if os.path.exists(gw_src):
        def gw(name):
            out = os.path.join(LIB, "mex", name + ".so")
            if _newer(out, [gw_src, so, shim] + headers):
                _run([CXX, "-O2", "-fPIC", "-shared", "-std=c++17", f"-DMLG_GATEWAY_{name}",
                      "-I", os.path.join(CSRC, "mexshim"), "-I", INCLUDE, "-o", out, gw_src,
                      "-L", LIB, "-lmonalisa_gpu", "-lmexshim", "-Wl,-rpath,$ORIGIN/.."])
        with ThreadPoolExecutor(jobs or min(8, os.cpu_count() or 4)) as ex:
            list(ex.map(gw, GATEWAYS))
    drv_src = os.path.join(ROOT, "driver", "monalisa_driver.cpp")
    drv = os.path.join(ROOT, "driver", "_bin", "monalisa_driver")
    if os.path.exists(drv_src) and _newer(drv, [drv_src, so] + headers):
        os.makedirs(os.path.dirname(drv), exist_ok=True)
        _run([CXX, "-O2", "-std=c++17", "-I", INCLUDE, "-I", os.path.join(CUDA_HOME, "include"), "-o", drv, drv_src,
              "-L", LIB, "-lmonalisa_gpu", "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart",
              "-Wl,-rpath,$ORIGIN/../../monalisa_b200/_lib", "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64")])
    if verbose:
        print("built", so)
    return so


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
