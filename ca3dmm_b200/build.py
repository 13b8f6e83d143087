"""Build libca3dmm_b200.so in-tree: C host engine (gcc) + sm_100a kernels (nvcc).

The library is the drop-in boundary: plain C ABI (include/*.h), no torch
types.  Run `python -m ca3dmm_b200.build` or call build().
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(ROOT, "include")
OBJ = os.path.join(HERE, "_obj")
LIB = os.path.join(HERE, "libca3dmm_b200.so")
ARCHIVE = os.path.join(HERE, "libca3dmm_b200.a")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

C_SOURCES = ["vcomm.c", "partition.c", "dev_type.c", "mat_redist.c", "cannon.c", "ca3dmm.c",
             "grouped.c", "autotune.c", "dist.c", "transport.c"]
CU_SOURCES = ["k_dgemm.cu", "k_pack.cu", "k_ozaki.cu", "k_crt.cu", "k_noalloc.cu", "k_mlp.cu",
              "k_tune_guard.cu"]
HEADERS = ["ca3dmm_kernels.h", "ca3dmm_ozaki.h", "ca3dmm_crt.h", "ca3dmm_util.h", "k_common.cuh",
           "k_split.cuh", "ca3dmm_tune_guard.h", "ca3dmm_tune_internal.h"]
EXAMPLES = ["example_cholesky_qr", "example_ab", "example_btb", "example_ab_dist"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(INC, f) for f in os.listdir(INC) if f.endswith(".h")]
    objs = []
    for src in C_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _newer(o, [s] + hdrs):
            _run(["gcc", "-O2", "-fPIC", "-std=gnu11", "-Wall", "-Wno-unused-function",
                  "-I", INC, "-I", CSRC, "-I", os.path.join(CUDA, "include"), "-c", s, "-o", o])
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _newer(o, [s] + hdrs):
            _run([NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                                  "-I", INC, "-I", CSRC, "-c", s, "-o", o])
    if _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs +
             ["-lm", "-lpthread", "-ldl"])
    # the static archive beside the shared library, as the reference installs both
    # (src/common.make:1-2, 56-66); link with -lcudart_static -lstdc++ -ldl -lpthread -lrt
    if _newer(ARCHIVE, objs):
        if os.path.exists(ARCHIVE):
            os.remove(ARCHIVE)
        _run(["ar", "rcs", ARCHIVE] + objs)
    # example callers (C programs linking the library like the reference's examples)
    for ex in EXAMPLES:
        s = os.path.join(HERE, "examples", ex + ".c")
        b = os.path.join(HERE, "examples", ex)
        if _newer(b, [s, LIB] + hdrs):
            _run(["gcc", "-O2", "-std=gnu11", "-I", INC, "-I", os.path.join(CUDA, "include"), s,
                  "-o", b, "-L", HERE, "-lca3dmm_b200", "-Wl,-rpath,$ORIGIN/..",
                  "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-lm", "-lpthread"])
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
