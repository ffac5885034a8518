"""The surrogate network's CPU oracle (oracle/mlp_oracle.py) against finite
differences of its own exact float64 forward pass, and its BF16 rounding
against known values.  The oracle is what the GPU gradient tests compare
with."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent.parent / "oracle"))
import mlp_oracle as M  # noqa: E402


def _master(seed):
    rng = np.random.default_rng(seed)
    m = np.zeros(M.PARAMS)
    for name, (o, n) in M.OFF.items():
        fan = {"W1": 64, "W5": 256, "Ws": 16}.get(name, 256)
        m[o:o + n] = rng.uniform(-1, 1, n) * np.sqrt(3.0 / fan)
    return m


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.14159265, 65504.0, 1e-40, 0.0])
    got = M.bf16(x)
    # 1 + 2^-8 is a tie: rounds to even (1.0); 1 + 1.5*2^-8 rounds up to 1 + 2^-7
    np.testing.assert_array_equal(got[:4], [1.0, 1.0, 1.0078125, 1.0078125])
    assert got[4] == -3.140625 and got[5] == 65536.0 and got[7] == 0.0


def test_split_features_reconstructs_to_16_bits():
    rng = np.random.default_rng(1)
    raw = rng.normal(size=(1000, 16)).astype(np.float32) * 7
    X = M.split_features(raw, np.zeros(16), np.ones(16))
    assert X.shape == (1000, 64)
    rel = np.abs(X[:, :16] + X[:, 16:32] - raw) / np.maximum(np.abs(raw), 1e-30)
    assert rel.max() < 2.0 ** -15


def test_exact_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    m = _master(3)
    X = rng.normal(size=(6, 64)) * 0.5
    dout = rng.normal(size=(6, 2))
    out, cache = M.forward(m, X, rounded=False)
    g = M.pack_grad(M.backward(cache, dout))

    def f(mm):
        return float((M.forward(mm, X, rounded=False)[0] * dout).sum())

    for name, (o, n) in M.OFF.items():
        for idx in rng.choice(n, size=min(3, n), replace=False):
            k = o + int(idx)
            h = 1e-5
            mp, mn = m.copy(), m.copy()
            mp[k] += h
            mn[k] -= h
            fd = (f(mp) - f(mn)) / (2 * h)
            assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (name, idx, fd, g[k])


def test_fourier_features_follow_their_definition():
    x = np.linspace(-1.9, 1.9, 301).astype(np.float32)
    f = M.fourier(x)
    for k in range(M.FREQ):
        np.testing.assert_allclose(f[:, 2 * k], np.sin(np.pi * 2.0 ** (k - 1) * x.astype(np.float64)), atol=1e-5)
        np.testing.assert_allclose(f[:, 2 * k + 1], np.cos(np.pi * 2.0 ** (k - 1) * x.astype(np.float64)), atol=1e-5)
