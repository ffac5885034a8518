"""The mixed-precision transfer's per-bin arithmetic, restated in numpy
float32 (each operation rounded to nearest, as the kernel's rounding
intrinsics do) and compared with the same sums in float64, on synthetic
rays of ~17,000 points: optically thin, bright, and optically thick ones
whose optical depth grows to ~1e13.  It pins the design of the five per-bin
values (an exact integer anchor S, Kahan pairs of tau log2(e) and of the
intensity scaled by 2^S; hadros_trace_kernel.cuh, bin_point/finish_pixel)
independently of the GPU: tau keeps ~1e-7 relative precision however large
the anchor, and the intensity ~1e-6, including the cases where earlier forms
of the accumulators failed (tau taken from one pair holding S - tau log2(e);
S recovered from that pair plus tau on thick rays)."""
from __future__ import annotations

import math

import numpy as np

F = np.float32
ANCHOR_MAX2 = F(57.70780)      # 40 / ln 2
UNDERFLOW2 = F(-1154.156)      # -800 / ln 2


def _kahan(s, c, x):
    y = F(x - c)
    t = F(s + y)
    c = F(F(t - s) - y)
    return t, c


def mixed_bin(args, ds):
    """args[i]: log2 of point i's emission term before attenuation (-inf: none);
    ds[i]: point i's absorption in log2 units (tau increment x log2 e).  Each
    point emits with the optical depth before it, then absorbs.  Returns
    (tau, I) as the kernel's finish forms them."""
    S = T = Tc = I = Ic = F(0.0)
    for arg, d in zip(args, ds):
        arg = F(arg)
        if arg != -np.inf and F(arg - F(T - Tc)) >= UNDERFLOW2:
            e = F(F(F(S - T) + arg) + Tc)
            if I == 0 or e > ANCHOR_MAX2:
                k = F(-np.rint(e))
                if I != 0:
                    sc = F(2.0) ** k
                    I, Ic = F(I * sc), F(Ic * sc)
                S = F(S + k)
                e = F(F(F(S - T) + arg) + Tc)
            I, Ic = _kahan(I, Ic, F(np.exp2(e)))
        T, Tc = _kahan(T, Tc, F(d))
    tau = (float(T) - float(Tc)) * math.log(2.0)
    inten = math.ldexp(float(I) - float(Ic), -int(S))
    return tau, inten


def exact_bin(args, ds):
    t2 = 0.0
    inten = 0.0
    for arg, d in zip(args, ds):
        if arg != -np.inf and arg - t2 >= -1154.156:
            inten += 2.0 ** (arg - t2)
        t2 += d
    return t2 * math.log(2.0), inten


def _ray(rng, n, log2_emission, d_scale, thick_from=None):
    """Smoothly varying emission exponents around log2_emission and positive
    absorption increments of scale d_scale; after point thick_from the
    absorption grows by twelve decades (a ray entering the dense torus)."""
    s = np.linspace(0.0, 6.0, n)
    args = log2_emission + 30.0 * np.sin(s) + rng.normal(0.0, 2.0, n)
    args[rng.random(n) < 0.05] = -np.inf          # points without emission
    ds = d_scale * np.exp(rng.normal(0.0, 1.0, n))
    if thick_from is not None:
        ds[thick_from:] *= 1e12
    return args.astype(np.float32), ds.astype(np.float32)


def _check(args, ds, rtol_tau, rtol_i):
    tau, inten = mixed_bin(args, ds)
    tau_x, inten_x = exact_bin(args.astype(np.float64), ds.astype(np.float64))
    assert abs(tau - tau_x) <= rtol_tau * tau_x, (tau, tau_x)
    assert abs(inten - inten_x) <= rtol_i * inten_x, (inten, inten_x)
    return tau_x, inten_x


def test_thin_ray_keeps_tau_and_intensity():
    rng = np.random.default_rng(1)
    args, ds = _ray(rng, 17000, -120.0, 1e-7)
    tau, inten = _check(args, ds, 1e-6, 1e-5)
    assert tau < 0.01 and inten > 0.0


def test_bright_ray_far_above_float32_range():
    """Emission terms of 2^300: the intensity itself is beyond FP32, the
    scaled sum and the anchor carry it."""
    rng = np.random.default_rng(2)
    args, ds = _ray(rng, 17000, 300.0, 1e-4)
    _, inten = _check(args, ds, 1e-6, 1e-5)
    assert inten > 1e90


def test_thick_ray_keeps_tau_relative_precision_and_the_anchor():
    """tau grows to ~1e13 behind the torus: S must stay the exact anchor of the
    intensity gathered before it (recovering it as rint((S - tau log2 e) + tau
    log2 e) from two FP32 pairs of that size gets it wrong by many units), and
    tau keep its relative precision."""
    rng = np.random.default_rng(3)
    args, ds = _ray(rng, 17000, -80.0, 1e-3, thick_from=8000)
    tau, inten = _check(args, ds, 1e-6, 1e-5)
    assert tau > 1e12 and inten > 0.0


def test_small_tau_behind_a_large_anchor():
    """The case that breaks tau = S - (S - tau log2 e): a faint, optically thin
    ray whose anchor is large (emission far below 1)."""
    rng = np.random.default_rng(4)
    args, ds = _ray(rng, 17000, -900.0, 1e-9)
    tau, _ = _check(args, ds, 1e-6, 1e-5)
    assert tau < 1e-4
