"""Cost-model MLP kernels against the CPU oracle, and the autotuner."""
import os
import tempfile

import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

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
    cands = [(0, 0, 1, 8, 0), (0, 0, 2, 8, 0), (0, 0, 4, 4, 0), (1, 7, 1, 8, 0),
             (1, 7, 2, 16, 0), (2, 0, 1, 32, 256), (2, 0, 1, 8, 128)]
    best, ms, err = cb.autotune(m, n, k, 0, 0, dA, lda, dB, ldb, dC, m, cands, with_err=True)
    # every candidate ran; split ones are timed or rejected by the guard
    assert np.all((ms > 0) | (ms == -2)) and np.all(err >= 0)
    assert np.all(ms[[0, 1, 2]] > 0)
    assert best == int(np.argmin(np.where(ms > 0, ms, np.inf)))
    cm = cb.CostModel(seed=11)
    best2, ms2 = cb.autotune(m, n, k, 0, 0, dA, lda, dB, ldb, dC, m, cands, model=cm, topk=2)
    assert int(np.sum(ms2 > 0)) == 2 and ms2[best2] > 0


def _oracle_c(A, B, m, n, k, cfg):
    """C of an engine configuration (1 x 1 x 1 grid): bit-exact oracles for the
    split modes, None for the plain mode (checked against the DD bound)."""
    mode, sl = cfg[0], cfg[1]
    if mode == cb.GEMM_CRT:
        P = orc.crt_bits(sl, k)
        c = orc.crt_gemm(np.asfortranarray(A), np.asfortranarray(B), 0, 0, m, n, k, P)
        return orc.nonfinite_fixup(np.asfortranarray(A), np.asfortranarray(B), 0, 0, m, n, k, c)
    if mode == cb.GEMM_OZAKI:
        qa, ea = orc.ozaki_slices_rows(np.asfortranarray(A), 0, m, k, sl)
        qb, eb = orc.ozaki_slices_cols(np.asfortranarray(B), 0, k, n, sl)
        return orc.ozaki_gemm(qa, ea, qb, eb, m, n, k, sl)
    return None


@pytest.mark.parametrize("tile", [128, 256])
def test_crt_tile_widths_bitexact(cuda, tile):
    """Both modular GEMM tile widths give the oracle's C bit for bit (edge tiles
    in both dimensions, bands of 8 and 32 tile rows)."""
    m, n, k = 1100, 700, 900
    A = orc.gen_signed_exp(31, m, k)
    B = orc.gen_signed_exp(32, k, n)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    want = _oracle_c(A, B, m, n, k, (cb.GEMM_CRT, 15))
    for band in (8, 32):
        dC = dev_zeros(m * n)
        e = cb.Ca3dmmEngine(m, n, k)
        assert e.set_tune((cb.GEMM_CRT, 15, 1, band, tile)) == 0
        assert e.get_tune() == (cb.GEMM_CRT, 15, 1, band, tile)
        assert e.exec(dA, lda, dB, ldb, dC, m) == 0
        got = from_dev(dC, m, n)
        e.free()
        assert np.array_equal(got, want), (band, np.max(np.abs(got - want)))


def test_set_tune_refusals(cuda):
    e = cb.Ca3dmmEngine(256, 256, 256)
    assert e.set_tune((cb.GEMM_CRT, 15, 1, 8, 64)) != 0        # no 64-column modular tile
    assert e.set_tune((cb.GEMM_PLAIN, 0, 1, 8, 96)) != 0       # plain tiles: 128 or 64 columns
    assert e.set_tune((cb.GEMM_OZAKI, 7, 1, 8, 64)) != 0       # the slice GEMM has one tile
    assert e.set_tune((cb.GEMM_PLAIN, 0, 1, 8, 128)) == 0
    assert e.get_tune() == (cb.GEMM_PLAIN, 0, 1, 8, 0)          # 0: the default width, 128
    assert e.set_tune((cb.GEMM_PLAIN, 0, 1, 8, 64)) == 0
    assert e.get_tune() == (cb.GEMM_PLAIN, 0, 1, 8, 64)
    assert e.set_tune((cb.GEMM_PLAIN, 0, 1, 5, 0)) != 0        # raster 4, 8 or 16
    assert e.set_tune((cb.GEMM_OZAKI, 9, 1, 8, 0)) != 0        # 2..8 slices
    assert e.set_tune((cb.GEMM_PLAIN, 0, 1, 16, 0)) == 0
    assert e.get_tune() == (cb.GEMM_PLAIN, 0, 1, 16, 0)


@pytest.mark.parametrize("how", [0, 1, 2])
def test_engine_auto_picks_the_tuned_config_and_matches_the_oracle(cuda, how):
    """An engine in auto mode tunes at its first exec: the configuration it
    keeps is the fastest admissible one of its report (exhaustive, model:
    among the timed ones; off: the model's first admissible), and its C is the
    oracle's for that configuration."""
    m, n, k = 1000, 900, 1200
    A = orc.gen_signed_exp(41, m, k, emin=-2, emax=2)
    B = orc.gen_signed_exp(42, k, n, emin=-2, emax=2)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k)
    assert e.set_gemm_mode(cb.GEMM_AUTO) == 0 and e.s.gemm_auto == 1
    import os
    old = os.environ.get("CA3DMM_AUTOTUNE")
    os.environ["CA3DMM_AUTOTUNE"] = ("off", "model", "exhaustive")[how]
    try:
        assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    finally:
        if old is None:
            del os.environ["CA3DMM_AUTOTUNE"]
        else:
            os.environ["CA3DMM_AUTOTUNE"] = old
    assert e.s.gemm_auto == 2 and e.s.tune_ms > 0
    rep = e.tune_report()
    chosen = e.get_tune()
    timed = [(ms, c) for c, ms, _ in rep if ms > 0]
    if how == 0:
        assert not timed
    else:
        assert timed and chosen == min(timed)[1]
        if how == 2:
            assert all(ms > 0 or ms == -2 for _, ms, _ in rep)
    # at this mild exponent spread every split candidate passes the guard
    assert all(ms != -2 for _, ms, _ in rep)
    got = from_dev(dC, m, n)
    want = _oracle_c(A, B, m, n, k, chosen)
    if want is not None:
        assert np.array_equal(got, want)
    else:
        hi, lo, ab = orc.dd_gemm(A, B, 0, 0, m, n, k)
        assert np.all(np.abs(got - hi) <= k * 2.0 ** -53 * ab + 1e-300)
    # later execs reuse the choice without tuning
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0 and e.get_tune() == chosen and e.s.n_exec == 2
    e.free()


def test_guard_rejects_split_precision_where_it_loses_accuracy(cuda):
    """Rows whose one large entry meets a zero row of B: their C entries come
    from entries 2^40 below the row maximum, which P-bit rounding below the
    maximum wipes out.  The guard rejects every split candidate; the engine
    keeps the plain GEMM."""
    m, n, k = 512, 384, 640
    rng = np.random.default_rng(5)
    A = rng.uniform(-1, 1, (m, k))
    B = rng.uniform(-1, 1, (k, n))
    spiky = rng.choice(m, 16, replace=False)
    A[spiky, 0] = 2.0 ** 40
    B[0, :] = 0.0
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k)
    rc, chosen = e.autotune(dA, lda, dB, ldb, dC, m, how=2)
    assert rc == 0
    rep = e.tune_report()
    assert all(ms == -2 for c, ms, _ in rep if c[0] != cb.GEMM_PLAIN), rep
    assert chosen[0] == cb.GEMM_PLAIN
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    hi, lo, ab = orc.dd_gemm(A, B, 0, 0, m, n, k)
    got = from_dev(dC, m, n)
    assert np.all(np.abs(got - hi) <= k * 2.0 ** -53 * ab + 1e-300)
    e.free()


def test_guard_rejects_split_on_nonfinite_operands(cuda):
    m, n, k = 256, 256, 300
    A = orc.gen_uniform(3, m, k)
    B = orc.gen_uniform(4, k, n)
    A[7, 11] = np.inf
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k)
    rc, chosen = e.autotune(dA, lda, dB, ldb, dC, m, how=2)
    assert rc == 0 and chosen[0] == cb.GEMM_PLAIN
    assert all(ms == -2 for c, ms, _ in e.tune_report() if c[0] != cb.GEMM_PLAIN)
    e.free()


def test_tune_cache_and_host_exec(cuda, tmp_path, monkeypatch):
    """CA3DMM_GEMM_MODE=auto with CA3DMM_TUNE_CACHE: the first engine tunes and
    appends its choice; a second engine of the same problem takes it from the
    cache (one report entry, no timing), here through exec_host."""
    import torch
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("CA3DMM_GEMM_MODE", "auto")
    monkeypatch.setenv("CA3DMM_TUNE_CACHE", str(cache))
    monkeypatch.setenv("CA3DMM_AUTOTUNE", "exhaustive")
    m, n, k = 700, 500, 800
    A = orc.gen_signed_exp(21, m, k, emin=-2, emax=2)
    B = orc.gen_signed_exp(22, k, n, emin=-2, emax=2)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e1 = cb.Ca3dmmEngine(m, n, k, p=4)
    assert e1.s.gemm_auto == 1
    assert e1.exec(dA, lda, dB, ldb, dC, m) == 0
    first = e1.get_tune()
    assert len(e1.tune_report()) > 1
    e1.free()
    line = cache.read_text().strip().splitlines()
    assert len(line) == 1 and line[0].startswith("v1 700 500 800 0 0 0 0 ")
    e2 = cb.Ca3dmmEngine(m, n, k, p=4)
    hA = torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).pin_memory()
    hB = torch.from_numpy(np.asfortranarray(B).ravel(order="F").copy()).pin_memory()
    hC = torch.zeros(m * n, dtype=torch.float64).pin_memory()
    assert e2.exec_host(hA, m, hB, k, hC, m) == 0
    assert e2.s.gemm_auto == 2 and e2.get_tune() == first
    assert len(e2.tune_report()) == 1
    got = np.asfortranarray(hC.numpy().reshape((m, n), order="F"))
    want = _oracle_c(A, B, m, n, k, first)
    if want is not None and e2.s.kp == 1:
        assert np.array_equal(got, want)
    hi, lo, ab = orc.dd_gemm(A, B, 0, 0, m, n, k)
    assert np.all(np.abs(got - hi) <= 2 * k * 2.0 ** -53 * ab + 1e-300)
    e2.free()


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


def test_engine_auto_btb(cuda):
    """B^T B in auto mode: the tuner sees op(A) = B^T (the guard samples B's
    columns on both sides) and the result stays within the plain GEMM's bound
    (the kept configuration passed the guard)."""
    n, k = 300, 20000
    Bm = orc.gen_btb(77, k, n)
    dB, ldb = to_dev(Bm)
    dC = dev_zeros(n * n)
    e = cb.Ca3dmmEngine(n, n, k, p=8, btb=True)
    assert e.set_gemm_mode(cb.GEMM_AUTO) == 0
    import os
    old = os.environ.get("CA3DMM_AUTOTUNE")
    os.environ["CA3DMM_AUTOTUNE"] = "exhaustive"
    try:
        assert e.exec(None, 0, dB, ldb, dC, n) == 0
    finally:
        if old is None:
            del os.environ["CA3DMM_AUTOTUNE"]
        else:
            os.environ["CA3DMM_AUTOTUNE"] = old
    assert e.s.gemm_auto == 2
    rep = e.tune_report()
    assert len(rep) > 1 and all(ms > 0 or ms == -2 for _, ms, _ in rep)
    got = from_dev(dC, n, n)
    hi, lo, ab = orc.dd_gemm(Bm, Bm, 1, 0, n, n, k)
    assert np.all(np.abs(got - hi) <= 2 * k * 2.0 ** -53 * ab + 1e-300)
    e.free()


@pytest.mark.parametrize("m,n,k,ta,tb,p", [(1, 1, 1, 0, 0, 1), (3, 700, 5, 1, 0, 2),
                                           (130, 2, 900, 0, 1, 3), (257, 129, 64, 1, 1, 6),
                                           (64, 64, 20000, 0, 0, 8)])
def test_engine_auto_small_and_odd_shapes(cuda, m, n, k, ta, tb, p):
    """Auto mode over degenerate and odd shapes: every candidate that runs
    gives a result the guard can assess, the kept one is admissible, and C is
    within the plain GEMM's bound."""
    A = orc.gen_signed_exp(51 + m, *((k, m) if ta else (m, k)), emin=-3, emax=3)
    B = orc.gen_signed_exp(52 + n, *((n, k) if tb else (k, n)), emin=-3, emax=3)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p)
    assert e.set_gemm_mode(cb.GEMM_AUTO) == 0
    rc, chosen = e.autotune(dA, lda, dB, ldb, dC, m, how=2)
    assert rc == 0
    rep = {c: ms for c, ms, _ in e.tune_report()}
    assert rep[chosen] > 0
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    got = from_dev(dC, m, n)
    hi, lo, ab = orc.dd_gemm(A, B, ta, tb, m, n, k)
    assert np.all(np.abs(got - hi) <= 2 * k * 2.0 ** -53 * ab + 1e-300)
    e.free()


def test_tune_cache_entry_this_engine_cannot_take(cuda, tmp_path, monkeypatch):
    """A cache line that does not fit the engine (a modular tile width that does
    not exist) is ignored: the engine tunes and appends its own choice."""
    m, n, k = 300, 200, 400
    e0 = cb.Ca3dmmEngine(m, n, k)
    key = "v1 %d %d %d 0 0 0 0 %d %d %d" % (m, n, k, e0.s.mp, e0.s.np, e0.s.kp)
    e0.free()
    cache = tmp_path / "tune.txt"
    cache.write_text(key + " : 2 15 32 64\n")
    monkeypatch.setenv("CA3DMM_GEMM_MODE", "auto")
    monkeypatch.setenv("CA3DMM_TUNE_CACHE", str(cache))
    monkeypatch.setenv("CA3DMM_AUTOTUNE", "exhaustive")
    A = orc.gen_signed_exp(61, m, k, emin=-2, emax=2)
    B = orc.gen_signed_exp(62, k, n, emin=-2, emax=2)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    assert e.s.gemm_auto == 2 and len(e.tune_report()) > 1
    lines = cache.read_text().strip().splitlines()
    assert len(lines) == 2 and lines[1].startswith(key)
    hi, lo, ab = orc.dd_gemm(A, B, 0, 0, m, n, k)
    assert np.all(np.abs(from_dev(dC, m, n) - hi) <= 2 * k * 2.0 ** -53 * ab + 1e-300)
    e.free()
