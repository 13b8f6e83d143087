"""Cost-model study: collect autotuner timings, train the MLP on the GPU with
the library's own CUDA kernels, and evaluate it against exhaustive search.

  python -m ca3dmm_b200.costmodel --train 1600 --test 400 --out DIR

Shapes: m, n, k log-uniform in [lo, hi] (default [128, 16384]), random
transposes, entries sign * (1 + u) * 2^e with e uniform in [-E, E], E drawn
per shape from {0, 4, 8} (the exponent-spread feature).  Candidates
(ca3dmm_tune_cfg_t: mode, slices or moduli, kp, raster or band, tile
columns): plain FP64 DMMA with k-slab splits kp in {1, 2, 4} and raster
bands of 8 or 16 tile rows on 128-column tiles, and on 64-column tiles with
raster 8; 7 INT8 slices with kp in {1, 2} and raster 8 or 16, and 8 slices;
the modular mode at the fewest moduli for 51-bit integers with 256- or
128-column tiles and bands of 32 or 8 tile rows, and at two moduli more (19
configurations).  Every candidate is timed on every shape on
one engine per kp (ca3dmm_engine_set_tune between candidates: one warm-up,
then the mean of `reps` execs from the engine's device events).  The MLP is
trained on log2(ms) of the training shapes and evaluated on the held-out
shapes by
  * regret = t(choice) / t(best) - 1 of the model's top-1 (no timing) and of
    the best of its top-2 (two timings),
  * search time saved = 1 - (time to time the top-2) / (time to time all),
against the untuned default (plain, kp = 1, raster 8).  Timing regret is
over all candidates: the accuracy guard that the engine's tuner puts in front
of split precision is a property of the data, not of the time.
"""
import argparse
import json
import os
import time

import numpy as np

import ca3dmm_b200 as cb

AUTO, AUTO2 = 0, -2    # the fewest moduli for 51-bit integers; two more
CANDS = ([(0, 0, kp, r, 0) for kp in (1, 2, 4) for r in (8, 16)] +
         [(0, 0, kp, 8, 64) for kp in (1, 2, 4)] +
         [(1, 7, kp, r, 0) for kp in (1, 2) for r in (8, 16)] + [(1, 8, 1, 8, 0)] +
         [(2, AUTO, 1, band, tn) for tn in (256, 128) for band in (32, 8)] +
         [(2, AUTO2, 1, 32, 256)])
DEFAULT = CANDS.index((0, 0, 1, 8, 0))


def crt_auto(k):
    """Moduli of the modular mode's automatic choice at depth k."""
    L = cb.lib()
    ns = (k + 131071) // 131072
    kmax = (k + ns - 1) // ns
    for nm in range(8, 19):
        if L.ca3dmm_crt_bits(nm, kmax) >= 51:
            return nm
    return 18


def resolve(c, k):
    """A study candidate with its moduli count made explicit for depth k."""
    mode, sl, kp, r, tn = c
    if mode == 2 and sl == AUTO2:
        sl = min(18, crt_auto(k) + 2)
    return (mode, sl, kp, r, tn)


def shapes(count, seed, lo, hi):
    rng = np.random.default_rng(seed)
    d = np.exp(rng.uniform(np.log(lo), np.log(hi), size=(count, 3))).round().astype(int)
    ta = rng.integers(0, 2, count)
    tb = rng.integers(0, 2, count)
    em = rng.choice([0, 4, 8], count)
    return [(int(a), int(b), int(c), int(x), int(y), int(e)) for (a, b, c), x, y, e in
            zip(d, ta, tb, em)]


def fill(buf, rows, cols, emax, gen):
    import torch
    n = rows * cols
    v = buf[:n]
    u = torch.rand(n, dtype=torch.float64, device="cuda", generator=gen)
    e = torch.randint(-emax, emax + 1, (n,), device="cuda", generator=gen).double()
    s = torch.randint(0, 2, (n,), device="cuda", generator=gen).double() * 2 - 1
    v.copy_(s * (1 + u) * torch.pow(2.0, e))
    return float(2 * emax + 1)


def time_cfg(eng, cfg, A, lda, B, ldb, Cm, m, reps):
    """Mean device time (ms) of `reps` execs under cfg after one warm-up."""
    if eng.set_tune(cfg) != 0:
        return float("nan")
    if eng.exec(A, lda, B, ldb, Cm, m) != 0:
        return float("nan")
    eng.reset_stat()
    for _ in range(reps):
        if eng.exec(A, lda, B, ldb, Cm, m) != 0:
            return float("nan")
    s = eng.s
    return (s.redist_ms + s.cannon_ms + s.reduce_ms) / max(1, s.n_exec)


def collect(shape_list, maxdim, reps=1, log_every=100):
    import torch
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234)
    A = torch.empty(maxdim * maxdim, dtype=torch.float64, device="cuda")
    B = torch.empty(maxdim * maxdim, dtype=torch.float64, device="cuda")
    Cm = torch.empty(maxdim * maxdim, dtype=torch.float64, device="cuda")
    feats, times = [], []
    t0 = time.time()
    for si, (m, n, k, ta, tb, em) in enumerate(shape_list):
        ar, ac = (k, m) if ta else (m, k)
        br, bc = (n, k) if tb else (k, n)
        spread = fill(A, ar, ac, em, gen)
        fill(B, br, bc, em, gen)
        row_f, row_t = [None] * len(CANDS), [float("nan")] * len(CANDS)
        for kp in sorted(set(c[2] for c in CANDS)):
            eng = None
            if kp <= k:
                eng = cb.Ca3dmmEngine(m, n, k, ta, tb, p=kp, proc_grid=(1, 1, kp))
            for ci, c in enumerate(CANDS):
                if c[2] != kp:
                    continue
                rc = resolve(c, k)
                row_f[ci] = cb.tune_features(m, n, k, ta, tb, rc, spread)
                if eng is not None and eng.ok:
                    row_t[ci] = time_cfg(eng, rc, A, ar, B, br, Cm, m, reps)
            if eng is not None:
                eng.free()
        feats.append(np.stack(row_f))
        times.append(np.array(row_t))
        if log_every and (si + 1) % log_every == 0:
            print("collected %d shapes in %.0f s" % (si + 1, time.time() - t0), flush=True)
    return np.stack(feats), np.stack(times)


def evaluate(model, F, T):
    ns, nc, nf = F.shape
    pred = model.predict(F.reshape(-1, nf)).reshape(ns, nc)
    ok = np.all(np.isfinite(T), axis=1)
    r1, r2, rdef, saved = [], [], [], []
    for i in np.nonzero(ok)[0]:
        best = np.min(T[i])
        order = np.argsort(pred[i])
        r1.append(T[i, order[0]] / best - 1)
        r2.append(min(T[i, order[0]], T[i, order[1]]) / best - 1)
        rdef.append(T[i, DEFAULT] / best - 1)
        saved.append(1 - (T[i, order[0]] + T[i, order[1]]) / np.sum(T[i]))
    q = lambda v: {"mean": float(np.mean(v)), "median": float(np.median(v)),
                   "p90": float(np.percentile(v, 90)), "max": float(np.max(v))}
    return {"shapes": int(len(r1)), "regret_model_top1": q(r1), "regret_model_top2": q(r2),
            "regret_untuned_default": q(rdef), "search_time_saved_top2": q(saved)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=1600)
    ap.add_argument("--test", type=int, default=400)
    ap.add_argument("--lo", type=int, default=128)
    ap.add_argument("--hi", type=int, default=16384)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--out", default="costmodel_out")
    ap.add_argument("--shipped", action="store_true",
                    help="also evaluate the shipped model (ca3dmm_b200/data) on the held-out shapes")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    tr = shapes(a.train, 11, a.lo, a.hi)
    te = shapes(a.test, 22, a.lo, a.hi)
    t0 = time.time()
    Ftr, Ttr = collect(tr, a.hi)
    Fte, Tte = collect(te, a.hi)
    t_collect = time.time() - t0
    np.savez_compressed(os.path.join(a.out, "costmodel_timings.npz"), Ftr=Ftr, Ttr=Ttr, Fte=Fte,
                        Tte=Tte)
    ok = np.isfinite(Ttr.ravel())
    X = Ftr.reshape(-1, Ftr.shape[-1])[ok]
    y = np.log2(Ttr.ravel()[ok]).astype(np.float32)
    model = cb.CostModel(seed=3)
    t1 = time.time()
    loss = model.train(X, y, epochs=a.epochs, batch=512, lr=2e-3)
    t_train = time.time() - t1
    model.save(os.path.join(a.out, "costmodel_b200.txt"))
    res = {"train_shapes": a.train, "test_shapes": a.test, "range": [a.lo, a.hi],
           "candidates": CANDS, "collect_s": t_collect, "train_s": t_train,
           "train_loss_log2ms": loss, "test": evaluate(model, Fte, Tte),
           "train": evaluate(model, Ftr, Ttr)}
    if a.shipped:
        res["shipped_test"] = evaluate(cb.CostModel.default(), Fte, Tte)
    with open(os.path.join(a.out, "costmodel_eval.json"), "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
