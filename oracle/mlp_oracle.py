"""CPU oracle of the surrogate network (test infrastructure only).

numpy float64 restatement of the forward and backward passes that the
library's training kernels (hadros_b200/csrc/hadros_mlp.cu) compute.  The
surrogate has no counterpart in the reference; this oracle restates the
network defined in hadros_b200/csrc/hadros_mlp.cuh so that the tests can
check the GPU gradients:

  X [n][64]    BF16 input columns: x_hi[16], x_lo[16], Fourier[32]
               (sin, cos of pi 2^(k-1) x for the normalized alpha and beta,
               k = 0..7); x = x_hi + x_lo
  Z1 = X W1d^T + b1          W1d = [W1f, W1f, W1four] (hi/lo weights tied)
  H_l = SiLU(Z_l), Z_{l+1} = H_l W_{l+1}^T + b_{l+1}   (l = 1..3)
  out = H4 W5^T + b5 + x Ws^T

With ``rounded=True`` the values are rounded to BF16 where the kernels store
BF16 (weights, Z_l, H_l, dZ_l) and SiLU is evaluated as the kernels do (from
h = bf16(Z_l) / 2 in BF16 arithmetic), so the GPU and the oracle differ only
by FP32 accumulation order and by the hardware tanh approximation.  With
``rounded=False`` it is the exact float64 network, whose gradient the tests
check against finite differences.
"""
from __future__ import annotations

import numpy as np

F, FREQ, W, DEPTH, OUT = 16, 8, 256, 4, 2
FOUR = 4 * FREQ
IN = 2 * F + FOUR

# FP32 master layout (hadros_mlp.cuh): W1 [256][48], b1, W2, b2, W3, b3, W4, b4,
# W5 [2][256], b5 [2], Ws [2][16].
OFF = {}
_o = 0
for _name, _size in (("W1", W * (F + FOUR)), ("b1", W), ("W2", W * W), ("b2", W), ("W3", W * W), ("b3", W),
                     ("W4", W * W), ("b4", W), ("W5", OUT * W), ("b5", OUT), ("Ws", OUT * F)):
    OFF[_name] = (_o, _size)
    _o += _size
PARAMS_USED = _o
PARAMS = (PARAMS_USED + 7) // 8 * 8
SHAPES = {"W1": (W, F + FOUR), "W2": (W, W), "W3": (W, W), "W4": (W, W), "W5": (OUT, W), "Ws": (OUT, F)}


def bf16(x) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float64).astype(np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    nan = np.isnan(f)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    out = u.astype(np.uint32).view(np.float32).astype(np.float64)
    return np.where(nan, np.nan, out)


def unpack(master: np.ndarray) -> dict:
    m = np.asarray(master, dtype=np.float64)
    d = {}
    for name, (o, n) in OFF.items():
        d[name] = m[o:o + n].reshape(SHAPES.get(name, (n,)))
    return d


def pack_grad(g: dict) -> np.ndarray:
    out = np.zeros(PARAMS)
    for name, (o, n) in OFF.items():
        out[o:o + n] = np.asarray(g[name]).reshape(-1)
    return out


def fourier(x: np.ndarray) -> np.ndarray:
    """[n] -> [n][16]: sin, cos of pi t, t = 2^(k-1) x reduced to [-1, 1]."""
    x = np.asarray(x, np.float32)
    out = []
    for k in range(FREQ):
        t = (x * np.float32(1 << k) * np.float32(0.5)).astype(np.float32)
        r = (t - np.float32(2.0) * np.rint(np.float32(0.5) * t)).astype(np.float32)
        a = np.pi * r.astype(np.float64)
        out += [np.sin(a), np.cos(a)]
    return np.stack(out, axis=1)


def split_features(raw: np.ndarray, mu: np.ndarray, inv_sd: np.ndarray) -> np.ndarray:
    """X [n][64] of k_featurize, as float64 BF16 values."""
    x = ((np.asarray(raw, np.float32) - np.asarray(mu, np.float32)) * np.asarray(inv_sd, np.float32))
    x = x.astype(np.float32)
    hi = bf16(x)
    lo = bf16(x.astype(np.float64) - hi)
    four = bf16(np.concatenate([fourier(x[:, 0]), fourier(x[:, 1])], axis=1))
    return np.concatenate([hi, lo, four], axis=1)


def silu(z):
    """z sigma(z) = h + h tanh(h), h = z / 2."""
    h = 0.5 * z
    return h + h * np.tanh(h)


def silu_bf16(z):
    """The kernels' SiLU: h = bf16(z) / 2, y = bf16(h + h * bf16(tanh h))."""
    h = 0.5 * bf16(z)
    return bf16(h + h * bf16(np.tanh(h)))


def silu_grad(z):
    h = 0.5 * z
    t = np.tanh(h)
    return 0.5 * (1.0 + t + h * (1.0 - t * t))


def forward(master, X, rounded: bool = True):
    """Returns (out [n][2], cache) for backward."""
    r = bf16 if rounded else (lambda a: np.asarray(a, dtype=np.float64))
    P = unpack(master)
    X = np.asarray(X, dtype=np.float64)
    x = X[:, :F] + X[:, F:2 * F]
    Wd = {1: r(np.concatenate([P["W1"][:, :F], P["W1"][:, :F], P["W1"][:, F:]], axis=1))}
    for l in (2, 3, 4):
        Wd[l] = r(P[f"W{l}"])
    W5 = r(P["W5"])
    Zs, Hs = {}, {0: X}
    for l in range(1, DEPTH + 1):
        z = Hs[l - 1] @ Wd[l].T + P[f"b{l}"]
        Zs[l] = r(z)
        Hs[l] = silu_bf16(z) if rounded else silu(z)
    out = Hs[DEPTH] @ W5.T + P["b5"] + x @ P["Ws"].T
    return out, {"Z": Zs, "H": Hs, "W": Wd, "W5": W5, "x": x, "r": r}


def backward(cache, dout) -> dict:
    """Gradient of sum(dout * out) in the master layout's blocks."""
    r = cache["r"]
    Z, H, Wd, W5, x = cache["Z"], cache["H"], cache["W"], cache["W5"], cache["x"]
    dout = np.asarray(dout, dtype=np.float64)
    g = {"W5": dout.T @ H[DEPTH], "b5": dout.sum(0), "Ws": dout.T @ x}
    dZ = r((dout @ W5) * silu_grad(Z[DEPTH]))
    for l in range(DEPTH, 1, -1):
        g[f"W{l}"] = dZ.T @ H[l - 1]
        g[f"b{l}"] = dZ.sum(0)
        dZ = r((dZ @ Wd[l]) * silu_grad(Z[l - 1]))
    gW1 = dZ.T @ H[0]
    g["W1"] = np.concatenate([gW1[:, :F] + gW1[:, F:2 * F], gW1[:, 2 * F:]], axis=1)
    g["b1"] = dZ.sum(0)
    return g
