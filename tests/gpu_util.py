"""Shared helpers for the GPU parity tests (seeded inputs, tolerances)."""
import numpy as np
import pytest


def need_gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def rand(rng, shape, dt, lo=-1.0, hi=1.0):
    return np.asfortranarray(rng.uniform(lo, hi, size=shape).astype(dt))


def tri_system(rng, side, m, n, dt, ld_pad=0):
    """Diagonally dominant triangular A (diag na + |N(0,1)|, off-diagonal N(0,1)/sqrt(na))
    and B ~ N(0,1) — the trsm input distribution of the benchmark configurations."""
    na = m if side in "Ll" else n
    a = rng.standard_normal((na + ld_pad, na)) / np.sqrt(na)
    a[np.arange(na), np.arange(na)] = na + np.abs(rng.standard_normal(na))
    b = rng.standard_normal((m + ld_pad, n))
    return np.asfortranarray(a.astype(dt)), np.asfortranarray(b.astype(dt)), na + ld_pad, m + ld_pad
