"""Builds the native library and executable of csu_b200 in-tree.

    csu_b200/lib/libcsu_b200.so   host C front end + CUDA engine (sm_100a), C ABI of include/csu_gpu.h
    csu_b200/bin/csu              drop-in solver executable (`csu <case dir>/`), same outputs as the
                                  reference executable

The CUDA code is compiled for sm_100a only, with --fmad=false and IEEE division/square root so that the
FP64 residual reproduces the reference's arithmetic; host C with -ffp-contract=off for the same reason.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
BIN_DIR = os.path.join(HERE, "bin")
OBJ_DIR = os.path.join(ROOT, "_build", "csu_b200")
LIB = os.path.join(LIB_DIR, "libcsu_b200.so")
EXE = os.path.join(BIN_DIR, "csu")

HOST_SOURCES = ["host/input.c", "host/su2.c", "host/case.c", "host/layout.c", "host/driver.c"]
CUDA_SOURCES = ["cuda/capi.cu", "cuda/noalloc.cu", "cuda/serve.cu"]
EXE_SOURCES = ["host/main.c"]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOSTCC = os.environ.get("CSU_HOSTCC", "gcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-std=c++17",
                     "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"]
CC_FLAGS = ["-O2", "-fPIC", "-std=gnu11", "-Wall", "-ffp-contract=off"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: %s" % os.path.basename(cmd[-1]))
    return r


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    out = [os.path.join(ROOT, "include", "csu_gpu.h")]
    for sub in ("host", "cuda"):
        d = os.path.join(SRC, sub)
        out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))]
    return out


def build(verbose=False, force=False):
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(BIN_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    inc = ["-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(SRC, "host"), "-I" + os.path.join(SRC, "cuda")]
    hdrs = _headers()
    objs = []
    for s in HOST_SOURCES:
        src = os.path.join(SRC, s)
        obj = os.path.join(OBJ_DIR, os.path.basename(s) + ".o")
        if force or _stale(obj, [src] + hdrs):
            _run([HOSTCC] + CC_FLAGS + inc + ["-c", src, "-o", obj])
        objs.append(obj)
    for s in CUDA_SOURCES:
        src = os.path.join(SRC, s)
        obj = os.path.join(OBJ_DIR, os.path.basename(s) + ".o")
        if force or _stale(obj, [src] + hdrs):
            _run([NVCC] + NVCC_FLAGS + inc + ["-c", src, "-o", obj])
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lm"])
    exe_objs = []
    for s in EXE_SOURCES:
        src = os.path.join(SRC, s)
        if not os.path.exists(src):
            continue
        obj = os.path.join(OBJ_DIR, os.path.basename(s) + ".o")
        if force or _stale(obj, [src] + hdrs):
            _run([HOSTCC] + CC_FLAGS + inc + ["-c", src, "-o", obj])
        exe_objs.append(obj)
    if exe_objs and (force or _stale(EXE, exe_objs + [LIB])):
        _run([HOSTCC, "-o", EXE] + exe_objs + ["-L" + LIB_DIR, "-lcsu_b200", "-Wl,-rpath,$ORIGIN/../lib", "-lm"])
    if verbose:
        print("built", LIB)
    return LIB


def ptxas_report():
    """Registers/spills of every kernel (-Xptxas -v), for tuning."""
    inc = ["-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(SRC, "host"), "-I" + os.path.join(SRC, "cuda")]
    r = subprocess.run([NVCC] + NVCC_FLAGS + inc + ["-Xptxas", "-v", "-c", os.path.join(SRC, "cuda", "capi.cu"),
                        "-o", os.devnull], capture_output=True, text=True)
    return r.stderr


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--ptxas":
        print(ptxas_report())
    else:
        build(verbose=True, force="--force" in sys.argv)
