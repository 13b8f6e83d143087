"""Build the CPU oracle (test infrastructure only).

  oracle/liboracle.so          -- oracle.c (double-double truth, geometry, slicing, MLP)
  oracle/_ref/libref_partition.so
                               -- the reference's own grid planner and balanced
                                  split, compiled unmodified from its sources
                                  (src/partition.c, src/utils.c) when the
                                  reference tree is present.  The rest of the
                                  reference needs MPI and CBLAS, which this
                                  image lacks, so only these two files build.
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
    return lib


if __name__ == "__main__":
    build()
    print("oracle built")
