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
REF = os.environ.get("CA3DMM_REFERENCE_DIR", "/root/reference")


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
    return lib


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
