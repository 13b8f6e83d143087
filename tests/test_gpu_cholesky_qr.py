"""The CholeskyQR caller (the reference's examples/example_CholeskyQR.c flow:
S = B^T B, R^-1 = inv(chol(S)), Q = B R^-1, check Q^T Q = I) built on the
engine, in both GEMM modes."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "ca3dmm_b200", "examples", "example_cholesky_qr")


def run(*args, env=None):
    r = subprocess.run([EXE] + [str(a) for a in args], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, **(env or {})))
    return r.returncode, r.stdout + r.stderr


def test_usage_without_gpu():
    rc, out = run(10, 20)            # nrow < ncol: rejected before any CUDA call
    assert rc == 1 and "usage" in out


def _err(out):
    m = re.search(r"CholeskyQR max error : ([0-9.e+-]+)", out)
    assert m, out
    return float(m.group(1))


@pytest.mark.gpu
@pytest.mark.parametrize("cond_exp", [0.0, 3.0])
def test_cholesky_qr_orthogonality(cuda, cond_exp):
    errs = {}
    for mode, sl in ((0, 0), (1, 7)):
        rc, out = run(60000, 256, mode, sl, 32, cond_exp)
        assert rc == 0, out
        errs[mode] = _err(out)
    assert errs[0] < 1e-12 and errs[1] < 1e-11, errs
    if cond_exp == 0:
        # split precision at 7 slices is no worse than twice the plain FP64 run
        assert errs[1] <= 2 * errs[0] + 1e-14, errs
    # with columns scaled over 10^+-1.5 a row of B spans three decades, and the
    # per-row exponent of the slicing leaves the small columns fewer bits: the
    # split result stays within 1e-11 but is not held to the plain error here


@pytest.mark.gpu
def test_cholesky_qr_symmetric_gram(cuda):
    """The Gram matrix through the symmetric B^T B (upper block triangle + mirror): the
    split-precision run gives the same error as the full product (same bits), the plain
    run stays as accurate."""
    for mode, sl in ((0, 0), (1, 7)):
        rc, full = run(60000, 256, mode, sl, 32, 0.0)
        assert rc == 0, full
        rc, sym = run(60000, 256, mode, sl, 32, 0.0, env={"CA3DMM_BTB_SYMMETRIC": "1"})
        assert rc == 0, sym
        if mode == 1:
            assert _err(sym) == _err(full), (full, sym)
        else:
            assert _err(sym) < 1e-12, sym
