"""Cost-model MLP kernels against the CPU oracle, and the autotuner."""
import os
import tempfile

import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, to_dev

pytestmark = pytest.mark.gpu


def test_mlp_gradients_match_oracle(cuda):
    rng = np.random.default_rng(1)
    nin, h1, h2, B = cb.NFEAT, 64, 64, 300
    cm = cb.CostModel(nin, h1, h2, seed=3)
    p = cm.params()
    X = rng.standard_normal((B, nin)).astype(np.float32)
    y = rng.standard_normal(B).astype(np.float32)
    loss, g = cm.fwd_bwd(X, y)
    loss_ref, _, g_ref = orc.mlp_fwd_bwd(p, X, y, nin, h1, h2)
    assert abs(loss - loss_ref) <= 1e-5 * max(1.0, abs(loss_ref))
    assert np.max(np.abs(g - g_ref)) <= 1e-4 * max(1.0, np.max(np.abs(g_ref)))


def test_mlp_training_fits_and_roundtrips(cuda):
    rng = np.random.default_rng(2)
    X = rng.uniform(0, 12, (2000, cb.NFEAT)).astype(np.float32)
    y = (0.3 * X[:, 0] + 0.2 * X[:, 1] * X[:, 2] / 12 - 0.1 * X[:, 5]).astype(np.float32)
    cm = cb.CostModel(seed=5)
    loss0, _ = cm.fwd_bwd((X - X.mean(0)) / X.std(0), y)
    loss = cm.train(X, y, epochs=150, batch=256, lr=3e-3)
    assert loss < 0.02 * loss0, (loss, loss0)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "m.txt")
        assert cm.save(path) == 0
        cm2 = cb.CostModel(path=path)
        assert np.allclose(cm.predict(X[:50]), cm2.predict(X[:50]), rtol=1e-5, atol=1e-5)


def test_autotune_exhaustive_and_model(cuda):
    m, n, k = 300, 260, 2000
    A = orc.gen_signed_exp(7, m, k)
    B = orc.gen_signed_exp(8, k, n)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    cands = [(0, 0, 1, 8), (0, 0, 2, 8), (0, 0, 4, 4), (1, 7, 1, 8), (1, 7, 2, 16)]
    best, ms = cb.autotune(m, n, k, 0, 0, dA, lda, dB, ldb, dC, m, cands)
    assert np.all(ms > 0)
    assert best == int(np.argmin(ms))
    cm = cb.CostModel(seed=11)
    best2, ms2 = cb.autotune(m, n, k, 0, 0, dA, lda, dB, ldb, dC, m, cands, model=cm, topk=2)
    assert int(np.sum(ms2 > 0)) == 2 and ms2[best2] > 0


def test_shipped_model_predicts_like_the_oracle(cuda):
    """The shipped model, loaded and run by the library's kernels, ranks the
    held-out study shapes exactly as the oracle's FP32 forward does."""
    from tests.test_costmodel_eval import TIMINGS, load_model
    nin, h1, h2, mu, sd, params = load_model()
    F = np.load(TIMINGS)["Fte"][:100]
    X = F.reshape(-1, nin)
    cm = cb.CostModel.default()
    got = cm.predict(X)
    Xn = ((X - mu) / sd).astype(np.float32)
    _, want, _ = orc.mlp_fwd_bwd(params, Xn, np.zeros(len(Xn), np.float32), nin, h1, h2)
    assert np.allclose(got, want, rtol=1e-4, atol=1e-4), np.max(np.abs(got - want))
