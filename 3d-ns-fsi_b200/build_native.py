"""Builds the native library of the package in-tree: 3d-ns-fsi_b200/lib/libnsfsi.so, and the reference-style
driver program 3d-ns-fsi_b200/bin/nsfsi_main (host/main.cpp).

CUDA sources are compiled by nvcc for sm_100a only; the host setup, config reader and C ABI are C++
compiled with -ffp-contract=off (the setup must reproduce the reference's floating-point expressions
exactly). The CUDA runtime is linked statically so the library carries no runtime-version dependency.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libnsfsi.so")
MAIN = os.path.join(PKG, "bin", "nsfsi_main")
BUILD = os.path.join(PKG, "_build")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["nsf_kernels.cu", "nsf_stage_ws.cu", "nsf_noalloc.cu", "nsf_adjoint.cu", "nsf_slab.cu"]
CXX_SOURCES = ["nsf_config.cpp", "nsf_setup.cpp", "nsf_capi.cpp", "nsf_ensemble.cpp", "nsf_adjoint.cpp", "nsf_bc_plan.cpp", "nsf_slab.cpp",
               "nsf_nccl.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("native build failed: " + os.path.basename(cmd[-1]))
    return r.stdout + r.stderr


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "nsfsi.h"))
    inc = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", *inc,
                   "-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            out = _run(cmd)
            if verbose or ptxas_info:
                print(out)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            _run(["g++", "-std=c++17", "-O3", "-ffp-contract=off", "-fPIC", "-Wall", *inc, "-I" + os.path.join(CUDA, "include"),
                  "-c", s, "-o", o])
    if _stale(LIB, objs):
        _run(["g++", "-shared", "-o", LIB, *objs, "-L" + os.path.join(CUDA, "lib64"), "-lcudart_static", "-ldl", "-lrt",
              "-lpthread", "-Wl,--no-undefined"])
    # the reference-style driver program (host/main.cpp over host/nsfsi_host.hpp)
    main_src = os.path.join(PKG, "host", "main.cpp")
    deps = [main_src, os.path.join(PKG, "host", "nsfsi_host.hpp"), os.path.join(ROOT, "include", "nsfsi.h"), LIB]
    if _stale(MAIN, deps):
        os.makedirs(os.path.dirname(MAIN), exist_ok=True)
        _run(["g++", "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(PKG, "host"),
              main_src, "-o", MAIN, "-L" + LIB_DIR, "-lnsfsi", "-Wl,-rpath,$ORIGIN/../lib", "-pthread"])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
