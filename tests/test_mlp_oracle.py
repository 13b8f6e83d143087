"""The MLP cost-model reference in the oracle is itself checked by finite
differences (CPU only)."""
import numpy as np

from oracle import oracle as orc


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    nin, h1, h2, B = 5, 7, 6, 9
    npar = h1 * nin + h1 + h2 * h1 + h2 + h2 + 1
    p = (rng.standard_normal(npar) * 0.5).astype(np.float32)
    X = rng.standard_normal((B, nin)).astype(np.float32)
    y = rng.standard_normal(B).astype(np.float32)
    loss, _, g = orc.mlp_fwd_bwd(p, X, y, nin, h1, h2)
    eps = 1e-2
    for idx in rng.choice(npar, 40, replace=False):
        pp, pm = p.copy(), p.copy()
        pp[idx] += eps
        pm[idx] -= eps
        fd = (orc.mlp_fwd_bwd(pp, X, y, nin, h1, h2)[0] - orc.mlp_fwd_bwd(pm, X, y, nin, h1, h2)[0]) / (2 * eps)
        assert abs(fd - g[idx]) <= 2e-2 * max(1.0, abs(fd)), (idx, fd, g[idx])
