"""Batched independent GEMMs in one grouped launch (plain and split precision),
including CUDA-graph capture and replay of the whole exec."""
import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

pytestmark = pytest.mark.gpu
U = 2.0 ** -53


def _batch(seed, nprob, lo=16, hi=700):
    rng = np.random.default_rng(seed)
    dims = np.exp(rng.uniform(np.log(lo), np.log(hi), size=(nprob, 3))).round().astype(int)
    ta = rng.integers(0, 2, nprob)
    tb = rng.integers(0, 2, nprob)
    probs = []
    for i, (m, n, k) in enumerate(dims):
        A = orc.gen_signed_exp(1000 + i, *((k, m) if ta[i] else (m, k)), emin=-4, emax=4, unit=True)
        B = orc.gen_signed_exp(2000 + i, *((n, k) if tb[i] else (k, n)), emin=-4, emax=4, unit=True)
        probs.append((int(m), int(n), int(k), int(ta[i]), int(tb[i]), A, B))
    return probs


def _upload(probs, even=False):
    dA, dB, dC, lda, ldb, ldc = [], [], [], [], [], []
    for m, n, k, ta, tb, A, B in probs:
        if even:     # even leading dimensions: operands in the launch's layout are read in place
            a, la = to_dev(A, pad_ld=A.shape[0] + (2 if A.shape[0] % 2 == 0 else 1))
            b, lb = to_dev(B, pad_ld=B.shape[0] + (2 if B.shape[0] % 2 == 0 else 1))
        else:        # odd pads exercise the pack path
            a, la = to_dev(A, pad_ld=A.shape[0] + 1)
            b, lb = to_dev(B)
        dA.append(a); lda.append(la); dB.append(b); ldb.append(lb)
        dC.append(dev_zeros(m * n)); ldc.append(m)
    return dA, dB, dC, lda, ldb, ldc


@pytest.mark.parametrize("mode,slices,even", [(cb.GEMM_PLAIN, 0, False), (cb.GEMM_PLAIN, 0, True),
                                              (cb.GEMM_OZAKI, 7, False)])
def test_grouped_batch(cuda, mode, slices, even):
    probs = _batch(5, 40)
    g = cb.GroupedGemm([p[0] for p in probs], [p[1] for p in probs], [p[2] for p in probs],
                       [p[3] for p in probs], [p[4] for p in probs], mode=mode, slices=slices)
    assert g.ok
    dA, dB, dC, lda, ldb, ldc = _upload(probs, even)
    assert g.exec(dA, lda, dB, ldb, dC, ldc) == 0
    for i, (m, n, k, ta, tb, A, B) in enumerate(probs):
        got = from_dev(dC[i], m, n)
        if mode == cb.GEMM_PLAIN:
            hi, lo, ab = orc.dd_gemm(A, B, ta, tb, m, n, k)
            assert np.max(np.abs(got - (hi + lo)) / ab) <= k * U, i
        else:
            opA = np.asfortranarray(A.T if ta else A)
            opB = np.asfortranarray(B.T if tb else B)
            qa, ea = orc.ozaki_slices_rows(opA, 0, m, k, slices)
            qb, eb = orc.ozaki_slices_cols(opB, 0, k, n, slices)
            assert np.array_equal(got, orc.ozaki_gemm(qa, ea, qb, eb, m, n, k, slices)), i


def test_grouped_cuda_graph_replay(cuda):
    import torch
    probs = _batch(9, 24)
    g = cb.GroupedGemm([p[0] for p in probs], [p[1] for p in probs], [p[2] for p in probs],
                       [p[3] for p in probs], [p[4] for p in probs])
    assert g.ok
    dA, dB, dC, lda, ldb, ldc = _upload(probs)
    assert g.exec(dA, lda, dB, ldb, dC, ldc) == 0        # plan uploaded, kernels warmed
    ref = [from_dev(c, p[0], p[1]) for c, p in zip(dC, probs)]
    for c in dC:
        c.zero_()
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    g.set_stream(s.cuda_stream, 0)
    with torch.cuda.graph(graph, stream=s):
        assert g.exec(dA, lda, dB, ldb, dC, ldc) == 0
    for _ in range(3):
        for c in dC:
            c.zero_()
        graph.replay()
        torch.cuda.synchronize()
        for i, p in enumerate(probs):
            assert np.array_equal(from_dev(dC[i], p[0], p[1]), ref[i]), i
    del graph


def test_grouped_rejects_bad_arguments(cuda):
    g = cb.GroupedGemm([10, 0], [10, 10], [10, 10])
    assert not g.ok
    g = cb.GroupedGemm([10], [10], [10], mode=cb.GEMM_OZAKI, slices=9)
    assert not g.ok
    g = cb.GroupedGemm([10], [10], [10])
    a, b, c = dev_zeros(100), dev_zeros(100), dev_zeros(100)
    assert g.exec([a], [9], [b], [10], [c], [10]) == 1        # ldA < m
