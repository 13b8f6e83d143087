"""The shipped cost model (ca3dmm_b200/data/costmodel_b200.txt) against
exhaustive autotuning on the 400 held-out shapes of the B200 study.

tests/golden/costmodel_timings_b200.npz holds the study's exhaustive timings
(every one of the 19 candidates -- plain at two tile widths, INT8-slice and modular
configurations with their k splits, rasters / bands and tile widths -- on
every shape, ms) and features, written by
  python -m ca3dmm_b200.costmodel --train 1600 --test 400 --epochs 300 --out DIR
on one B200.  The network is evaluated here with the oracle's FP32 forward.
What the network gains is measured against the tuner without it: the untuned
default, the best single configuration of the training shapes, and linear /
quadratic least-squares predictors on the same features.
"""
import os

import numpy as np
import pytest

from oracle import oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
MODEL = os.path.join(ROOT, "ca3dmm_b200", "data", "costmodel_b200.txt")
TIMINGS = os.path.join(HERE, "golden", "costmodel_timings_b200.npz")


def load_model(path=MODEL):
    lines = open(path).read().split("\n")
    hdr = lines[0].split()
    assert hdr[:2] == ["ca3dmm-mlp", "v1"]
    nin, h1, h2 = int(hdr[2]), int(hdr[3]), int(hdr[4])
    mu = np.array(lines[1].split(), dtype=np.float32)
    sd = np.array(lines[2].split(), dtype=np.float32)
    params = np.array([float(x) for x in lines[3:] if x.strip()], dtype=np.float32)
    return nin, h1, h2, mu, sd, params


@pytest.fixture(scope="module")
def study():
    z = np.load(TIMINGS)
    nin, h1, h2, mu, sd, params = load_model()

    def mlp(F):
        X = ((F.reshape(-1, nin) - mu) / sd).astype(np.float32)
        _, yhat, _ = orc.mlp_fwd_bwd(params, X, np.zeros(len(X), np.float32), nin, h1, h2)
        return yhat.reshape(F.shape[:2])

    return {"Ftr": z["Ftr"], "Ttr": z["Ttr"], "Fte": z["Fte"], "Tte": z["Tte"], "mlp": mlp,
            "mu": mu, "sd": sd, "nin": nin}


def regret(pred, T, top=1):
    ok = np.all(np.isfinite(T), axis=1)
    out = []
    for i in np.nonzero(ok)[0]:
        o = np.argsort(pred[i], kind="stable")[:top]
        out.append(T[i, o].min() / T[i].min() - 1.0)
    return np.array(out)


def lstsq_predictor(study, quadratic):
    mu, sd, nin = study["mu"], study["sd"], study["nin"]

    def design(F):
        X = (F.reshape(-1, nin) - mu) / sd
        cols = [X]
        if quadratic:
            iu = np.triu_indices(nin)
            cols.append((X[:, :, None] * X[:, None, :])[:, iu[0], iu[1]])
        cols.append(np.ones((len(X), 1)))
        return np.concatenate(cols, axis=1)

    y = np.log2(study["Ttr"].ravel())
    ok = np.isfinite(y)
    w, *_ = np.linalg.lstsq(design(study["Ftr"])[ok], y[ok], rcond=None)
    return (design(study["Fte"]) @ w).reshape(study["Tte"].shape)


def test_model_layout():
    nin, h1, h2, mu, sd, params = load_model()
    assert (nin, h1, h2) == (14, 64, 64)
    assert params.size == h1 * nin + h1 + h2 * h1 + h2 + h2 + 1
    assert np.all(sd > 0)


def test_held_out_regret_and_search_time(study):
    T = study["Tte"]
    P = study["mlp"](study["Fte"])
    r1, r2 = regret(P, T, 1), regret(P, T, 2)
    assert len(r1) == 400
    assert r1.mean() <= 0.03 and np.median(r1) <= 0.01, (r1.mean(), np.median(r1))
    assert r2.mean() <= 0.015 and np.median(r2) == 0.0, (r2.mean(), np.median(r2))
    # timing the model's top 2 instead of all 19 candidates
    order = np.argsort(P, axis=1)[:, :2]
    saved = 1.0 - np.take_along_axis(T, order, 1).sum(1) / T.sum(1)
    assert saved.mean() >= 0.85, saved.mean()


def test_network_beats_the_tuner_without_it(study):
    T = study["Tte"]
    r_mlp = regret(study["mlp"](study["Fte"]), T).mean()
    ncand = T.shape[1]
    default = regret(np.tile(np.arange(ncand) != 0, (len(T), 1)).astype(float), T).mean()
    Ttr = study["Ttr"][np.all(np.isfinite(study["Ttr"]), axis=1)]
    fixed_cfg = int(np.argmin(np.log(Ttr / Ttr.min(1, keepdims=True)).mean(0)))
    fixed = regret(np.tile(np.arange(ncand) != fixed_cfg, (len(T), 1)).astype(float), T).mean()
    linear = regret(lstsq_predictor(study, False), T).mean()
    quad = regret(lstsq_predictor(study, True), T).mean()
    print("\nmean top-1 regret on 400 held-out shapes: mlp %.4f, quadratic %.4f, linear %.4f, "
          "best fixed (cfg %d) %.4f, untuned default %.4f" % (r_mlp, quad, linear, fixed_cfg,
                                                               fixed, default))
    assert default >= 0.5
    assert r_mlp <= 0.2 * fixed and r_mlp <= 0.2 * linear
    assert r_mlp <= 0.6 * quad


def test_prediction_error(study):
    P = study["mlp"](study["Fte"])
    err = P - np.log2(study["Tte"])
    rmse = float(np.sqrt(np.nanmean(err ** 2)))
    assert rmse <= 0.15, rmse      # log2(ms): about 11 % per configuration
