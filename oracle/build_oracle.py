"""Build the CPU oracle (test infrastructure only).

  oracle/liboracle.so          -- oracle.c (double-double truth, geometry, slicing, MLP)
  oracle/_ref/libref_partition.so
                               -- the reference's own grid planner and balanced
                                  split, compiled unmodified from its sources
                                  (src/partition.c, src/utils.c) when the
                                  reference tree is present;
  oracle/_ref/libref_ca3dmm.so -- the reference's whole CPU path (src/ca3dmm.c,
                                  cannon.c, mat_redist.c, partition.c, utils.c,
                                  dev_type.c, mpi_op_omp.c), compiled unmodified
                                  against vmpi (oracle/vmpi: MPI ranks as host
                                  threads) and the OpenBLAS shipped in this
                                  image, plus the driver oracle/vmpi/ref_driver.c.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference tree: CA3DMM_REFERENCE_DIR, else a checkout named "reference" beside the repo.
REF = os.environ.get("CA3DMM_REFERENCE_DIR",
                     os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))


def _newer(t, deps):
    return not os.path.exists(t) or any(os.path.getmtime(d) > os.path.getmtime(t) for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("oracle build failed")


def build():
    src = os.path.join(HERE, "oracle.c")
    lib = os.path.join(HERE, "liboracle.so")
    if _newer(lib, [src]):
        # -ffp-contract=off: the double-double steps must not be fused.
        _run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", src, "-o", lib,
              "-lm"])
    refsrc = os.path.join(REF, "src")
    if os.path.isdir(refsrc):
        out = os.path.join(HERE, "_ref")
        os.makedirs(out, exist_ok=True)
        rlib = os.path.join(out, "libref_partition.so")
        deps = [os.path.join(refsrc, f) for f in ("partition.c", "utils.c", "partition.h", "utils.h")]
        if _newer(rlib, deps):
            _run(["gcc", "-O2", "-fPIC", "-shared", "-I", refsrc, deps[0], deps[1], "-o", rlib, "-lm"])
        openblas = find_openblas()
        if openblas:
            vdir = os.path.join(HERE, "vmpi")
            srcs = [os.path.join(refsrc, f) for f in ("ca3dmm.c", "cannon.c", "mat_redist.c",
                                                        "partition.c", "utils.c", "dev_type.c",
                                                        "mpi_op_omp.c")]
            mine = [os.path.join(vdir, f) for f in ("vmpi.c", "ref_driver.c")]
            hdrs = [os.path.join(vdir, f) for f in ("mpi.h", "cblas.h", "lapacke.h")]
            clib = os.path.join(out, "libref_ca3dmm.so")
            if _newer(clib, srcs + mine + hdrs):
                d, f = os.path.split(openblas)
                pre = ["-DVMPI_SCIPY_OPENBLAS"] if "scipy_openblas" in f else []
                _run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-DUSE_OPENBLAS"] + pre + [
                      "-Wno-implicit-function-declaration", "-I", vdir, "-I", refsrc] + srcs + mine +
                     ["-o", clib, "-L", d, "-l:" + f, "-Wl,--disable-new-dtags", "-Wl,-rpath," + d,
                      "-Wl,-Bsymbolic",
                      "-lpthread", "-lm"])
            build_ref_cuda(refsrc, out, vdir, openblas)
    return lib


# The reference's cuBLAS wrappers that touch its static handle; cuda_proxy.cu is
# compiled with each renamed, and ref_cuda_serial.c puts a lock in front.
_SERIALISED = ("cuda_cublas_dcopy", "cuda_cublas_dscal", "cuda_cublas_ddot", "cuda_cublas_dgemm",
               "cuda_cublas_dgeam", "cuda_cublas_dtrsm", "cuda_cusolver_dpotrf",
               "cuda_cusolver_dsyevd")


def build_ref_cuda(refsrc, out, vdir, openblas):
    """oracle/_ref/libref_ca3dmm_cuda.so: the reference's GPU path (USE_CUDA;
    src/cuda_proxy.cu rebuilt for sm_100a, linked to this image's cuBLAS,
    cuSOLVER and cuRAND) under vmpi, driven by ref_driver_cuda.c.  Context
    figures only; skipped when nvcc or the CUDA libraries are missing."""
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    nvcc = os.path.join(cuda, "bin", "nvcc")
    libdir = os.path.join(cuda, "lib64")
    if not (os.path.exists(nvcc) and os.path.exists(os.path.join(libdir, "libcublas.so"))):
        return None
    srcs = [os.path.join(refsrc, f) for f in ("ca3dmm.c", "cannon.c", "mat_redist.c", "partition.c",
                                                "utils.c", "dev_type.c", "mpi_op_omp.c")]
    cu = os.path.join(refsrc, "cuda_proxy.cu")
    mine = [os.path.join(vdir, f) for f in ("vmpi.c", "ref_driver_cuda.c", "ref_cuda_serial.c")]
    hdrs = [os.path.join(vdir, f) for f in ("mpi.h", "cblas.h", "lapacke.h")]
    clib = os.path.join(out, "libref_ca3dmm_cuda.so")
    if not _newer(clib, srcs + [cu] + mine + hdrs + [os.path.abspath(__file__)]):
        return clib
    obj = os.path.join(out, "ref_cuda_proxy.o")
    _run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-Xcompiler", "-fPIC",
          "-I", refsrc] + ["-D%s=vgpu_raw_%s" % (f, f) for f in _SERIALISED] + ["-c", cu, "-o", obj])
    d, f = os.path.split(openblas)
    pre = ["-DVMPI_SCIPY_OPENBLAS"] if "scipy_openblas" in f else []
    _run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-DUSE_OPENBLAS", "-DUSE_CUDA"] + pre + [
          "-Wno-implicit-function-declaration", "-I", vdir, "-I", refsrc,
          "-I", os.path.join(cuda, "include")] + srcs + mine + [obj] +
         ["-o", clib, "-L", d, "-l:" + f, "-L", libdir, "-lcublas", "-lcusolver", "-lcurand",
          "-lcudart", "-Wl,--disable-new-dtags", "-Wl,-rpath," + d, "-Wl,-rpath," + libdir,
          "-Wl,-Bsymbolic", "-lpthread", "-lm"])
    return clib


def find_openblas():
    """An LP64 OpenBLAS shipped in this image: the scipy wheel's build
    (0.3.31, scipy_-prefixed exports, Skylake-X kernels) first, else one with
    plain CBLAS names."""
    import glob
    import site
    for sp in site.getsitepackages():
        for pat in ("scipy.libs/libscipy_openblas-*.so", "opencv_python_headless.libs/libopenblas*.so*",
                    "*/libopenblas*.so*"):
            hits = sorted(glob.glob(os.path.join(sp, pat)))
            if hits:
                return hits[0]
    return None


if __name__ == "__main__":
    build()
    print("oracle built")
