"""Deferred transfer (HADROS_TRANSFER_DEFERRED): the trace kernel buffers each
ray's path points and the warp replays them into the bins, instead of every
thread adding each point to its ray's bins as it goes.  Same per-bin
arithmetic in the same point order: with the reference geodesic arithmetic
(no FMA contraction) every output must be the same bits as the in-loop
transfer's, for any bin count, for batches whose cameras have different bin
counts, and for plans.  With the fast arithmetic the two kernels are separate
compilations whose FMA contraction may differ (a ray's step count can move by
one, as between the fast kernel and the oracle), so there they are compared
with the mixed-precision tolerance."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("tau", "P_surv", "I_obs", "fate", "steps", "attempts", "tau_E", "I_E")


def _both(ctx, fn):
    try:
        ctx.set_transfer("in_loop")
        a = fn()
        ctx.set_transfer("deferred")
        b = fn()
    finally:
        ctx.set_transfer("auto")
    return a, b


def _same(a, b, what):
    for k in KEYS:
        if k in a:
            np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]), err_msg=f"{what}: {k}")


@pytest.mark.parametrize("workload,bins,nx,ny", [
    ("mixed_512", 8, 40, 32),
    ("mixed_512", 12, 33, 21),
    ("production_point", 16, 24, 24),
    ("production_point", 64, 24, 20),
    ("production_point", 80, 16, 16),
    ("mixed_512", 1, 48, 40),
])
def test_deferred_equals_in_loop(hb, gpu_ctx, sigma_table, workload, bins, nx, ny):
    from hadros_b200 import workloads as W
    kw = getattr(W, workload)(nx=nx, ny=ny, h=0.05, fast=False)
    kw.update(spectral="monochromatic") if bins == 1 else kw.update(n_bins=bins)
    p = hb.params(**kw)
    a, b = _both(gpu_ctx, lambda: gpu_ctx.image(p, sigma_table))
    _same(a, b, f"{workload} {bins} bins")
    assert np.isfinite(a["tau"]).all() and (a["steps"] > 0).all()


def test_deferred_batch_of_mixed_bin_counts(hb, gpu_ctx, sigma_table):
    from hadros_b200 import workloads as W
    cams = [hb.params(**W.mixed_512(nx=20, ny=18, h=0.05, n_bins=8, fast=False)),
            hb.params(**W.production_point(nx=16, ny=22, h=0.05, n_bins=24, fast=False)),
            hb.params(**W.mixed_512(nx=25, ny=9, h=0.05, spectral="monochromatic", fast=False))]
    a, b = _both(gpu_ctx, lambda: gpu_ctx.batch(cams, sigma_table))
    for k, (x, y) in enumerate(zip(a, b)):
        _same(x, y, f"camera {k}")


def test_deferred_plan_equals_batch(hb, gpu_ctx, sigma_table):
    """A plan built in deferred mode (auto picks it at 32 bins) traces what
    hadros_batch traces with the in-loop transfer."""
    import torch
    from hadros_b200 import workloads as W
    torch.cuda.set_device(0)
    cams = [hb.params(**W.production_point(nx=20, ny=20, h=0.05, n_bins=32, theta_obs_deg=t, fast=False))
            for t in (20.0, 60.0)]
    gpu_ctx.set_transfer("in_loop")
    try:
        ref = gpu_ctx.batch(cams, sigma_table)
    finally:
        gpu_ctx.set_transfer("auto")
    plan = gpu_ctx.plan(cams, sigma_table)
    out = plan.alloc(torch, device=torch.device("cuda", 0))
    plan.launch(out)
    torch.cuda.synchronize()
    o, ob = 0, 0
    for c, r in zip(cams, ref):
        P, B = c.nx * c.ny, c.n_bins
        for k in ("tau", "P_surv", "I_obs", "steps"):
            np.testing.assert_array_equal(out[k][o:o + P].cpu().numpy(), r[k], err_msg=k)
        np.testing.assert_array_equal(out["I_E"][ob:ob + P * B].cpu().numpy(), r["I_E"].reshape(-1))
        o += P
        ob += P * B
    plan.close()


@pytest.mark.parametrize("bins", [8, 64])
def test_fast_deferred_within_tolerance_of_in_loop(hb, gpu_ctx, sigma_table, bins):
    from hadros_b200 import workloads as W
    from parity import RTOL_MIXED, assert_parity
    p = hb.params(**W.production_point(nx=24, ny=20, h=0.05, n_bins=bins))
    assert p.fast_geodesic == 1
    a, b = _both(gpu_ctx, lambda: gpu_ctx.image(p, sigma_table))
    # rays whose step count moved (FMA contraction) are compared by fate only
    same = a["steps"] == b["steps"]
    np.testing.assert_array_equal(a["fate"], b["fate"])
    assert same.mean() >= 0.99 and np.abs(a["steps"] - b["steps"]).max() <= 1
    sub = lambda d: {k: v[same] for k, v in d.items()}
    assert_parity(sub(b), sub(a), RTOL_MIXED, f"fast deferred {bins} bins", p_absolute=True)


def test_deferred_128_bins_matches_the_oracle(hb, gpu_ctx, sigma_table, sigma_arrays):
    """128 bins: more than the in-loop transfer's shared memory holds (it
    reports HADROS_E_ARG/E_CUDA there); the deferred transfer (what auto picks)
    matches the CPU oracle within the mixed-precision tolerance."""
    from hadros_b200 import workloads as W
    from oracle import pyoracle as O
    from parity import RTOL_MIXED, assert_parity
    E, g2, s = sigma_arrays
    p = hb.params(**W.production_point(nx=6, ny=5, h=0.05, n_bins=128))
    ref = O.oracle_image(p, E, s)
    got = gpu_ctx.image(p, sigma_table)
    assert_parity(got, ref, RTOL_MIXED, "deferred 128 bins/mixed", p_absolute=True)
