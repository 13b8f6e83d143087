"""Test helpers: column-major host <-> device transfer through torch."""
import numpy as np


def to_dev(X, pad_ld=None):
    """Column-major copy of X on cuda:0 as a flat float64 tensor; returns (tensor, ld)."""
    import torch
    X = np.asfortranarray(X, dtype=np.float64)
    r, c = X.shape
    ld = pad_ld or r
    buf = np.zeros((ld, c), order="F")
    buf[:r, :] = X
    t = torch.from_numpy(buf.ravel(order="F").copy()).cuda()
    return t, ld


def from_dev(t, r, c, ld=None):
    ld = ld or r
    h = t.cpu().numpy()[: ld * c].reshape((ld, c), order="F")
    return np.asfortranarray(h[:r, :])


def dev_zeros(n):
    import torch
    return torch.zeros(max(int(n), 1), dtype=torch.float64, device="cuda")
