"""The reference's own GPU path (src/*.c with USE_CUDA, src/cuda_proxy.cu rebuilt
for sm_100a, DEV_TYPE_CUDA) on vmpi rank threads sharing this GPU: the context
figures beside the bench come from it, so it must compute the right product.
Each run is a child process (the reference ends its process on a CUDA error),
and its C is checked against the reference's CPU path under the reference's
own validation rule (componentwise relative difference <= 1e-12,
examples/example_AB.c:262-304) and against the GPU engine's plain FP64 result
within k u |A||B|."""
import os
import subprocess
import sys

import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_ca3dmm_cuda.so")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(LIB), reason="reference GPU path not built"),
              pytest.mark.skipif(orc.ref_lib() is None, reason="reference CPU path not built")]
U = 2.0 ** -53

CHILD = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
from oracle import oracle as orc
p, m, n, k, ta, tb, btb = (int(x) for x in sys.argv[2:9])
A = np.load(sys.argv[9]) if not btb else None
B = np.load(sys.argv[10])
grid = None if sys.argv[12] == "auto" else tuple(int(x) for x in sys.argv[12].split("x"))
C, times, g = orc.ref_ca3dmm_cuda(p, m, n, k, ta, tb, A, B, grid=grid, ntest=2, btb=bool(btb),
                                  timeout=120.0)
assert np.all(times > 0), times
np.save(sys.argv[11], C)
print("GRID %d %d %d %d" % g)
"""


def _ref_gpu(tmp_path, p, m, n, k, ta, tb, A, B, btb=False, grid=None):
    fa, fb, fc = (str(tmp_path / x) for x in ("a.npy", "b.npy", "c.npy"))
    if A is not None:
        np.save(fa, np.asfortranarray(A))
    np.save(fb, np.asfortranarray(B))
    gs = "auto" if grid is None else "x".join(str(x) for x in grid)
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(p), str(m), str(n), str(k), str(ta),
                        str(tb), str(int(btb)), fa, fb, fc, gs],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "[ERROR]" not in r.stderr, r.stderr[-2000:]
    g = tuple(int(x) for x in r.stdout.split("GRID")[1].split()[:4])
    return np.load(fc), g


def _rule_1e12(got, want, scale):
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
    bad = (rel > 1e-12) & (np.abs(got - want) > 1e-15 * scale)
    assert not bad.any(), (int(bad.sum()), float(rel.max()))


@pytest.mark.parametrize("m,n,k,ta,tb,p,grid", [
    (600, 500, 400, 0, 0, 4, None),
    (700, 300, 900, 1, 0, 6, None),
    (1024, 1024, 2048, 0, 1, 24, (4, 2, 3)),       # Cannon local k 341: one DGEMM per shift
])
def test_reference_gpu_path_product(cuda, tmp_path, m, n, k, ta, tb, p, grid):
    A = orc.gen_uniform(11, *((k, m) if ta else (m, k)))
    B = orc.gen_uniform(12, *((n, k) if tb else (k, n)))
    Cg, g = _ref_gpu(tmp_path, p, m, n, k, ta, tb, A, B, grid=grid)
    Cc, _, _, gc = orc.ref_ca3dmm(p, m, n, k, ta, tb, A, B, grid=grid)
    assert g == gc
    opA, opB = (A.T if ta else A), (B.T if tb else B)
    scale = np.abs(opA) @ np.abs(opB)
    _rule_1e12(Cg, Cc, scale)
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p, proc_grid=grid)
    assert e.ok and e.set_gemm_mode(cb.GEMM_PLAIN) == 0
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    ours = from_dev(dC, m, n)
    assert np.all(np.abs(ours - Cg) <= 2 * k * U * scale)


def test_reference_gpu_path_btb(cuda, tmp_path):
    n, k, p = 96, 4000, 8
    Bm = orc.gen_btb(21, k, n)
    Cg, g = _ref_gpu(tmp_path, p, n, n, k, 0, 0, None, Bm, btb=True, grid=(1, 1, 8))
    assert g[:3] == (1, 1, 8)
    Cc, _, _, _ = orc.ref_ca3dmm(p, n, n, k, 0, 0, None, Bm, grid=(1, 1, 8), btb=True)
    _rule_1e12(Cg, Cc, np.abs(Bm.T) @ np.abs(Bm))


def test_reference_gpu_path_kstack_defect(cuda, tmp_path):
    """Where the reference's Cannon stacks k panels before a DGEMM (local k below
    160 with np_dim > 1: gemm_cycle > 1, src/cannon.c:86-99), its GPU branch
    stacks into the host panels (A_stack_h, B_stack_h: src/cannon.c:459-463)
    but multiplies the device ones (A_stack_d, B_stack_d: :574-580), which were
    never written (fresh device memory: C comes back zero).  The CPU branch is right; so is the
    engine.  The bench's workloads (8000^3 on 4x2x3: local k 1334; B^T B on
    1x1x32: np_dim 1) stay outside this case."""
    m = n = k = 512
    A = orc.gen_uniform(13, m, k)
    B = orc.gen_uniform(14, k, n)
    Cg, g = _ref_gpu(tmp_path, 24, m, n, k, 0, 0, A, B, grid=(4, 2, 3))
    assert g[:3] == (4, 2, 3)
    assert not np.allclose(Cg, A @ B)
    e = cb.Ca3dmmEngine(m, n, k, 0, 0, p=24, proc_grid=(4, 2, 3))
    assert e.ok and e.set_gemm_mode(cb.GEMM_PLAIN) == 0
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    assert np.all(np.abs(from_dev(dC, m, n) - A @ B) <= 2 * k * U * (np.abs(A) @ np.abs(B)))
