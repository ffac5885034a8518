"""What the trained surrogate gains over the exact tracer alone.

A small ensemble (2 networks) is trained on rays that the tracer traces at
48 points of the production box (collapsar_ndaf_like, density_weighted
source, a = 0.95, rho0 in [1e9, 1e12], inclination in [10, 80] deg), at
512 x 512 pixels and 16 bins.  On a held-out point the surrogate image with
its exact fallback (pixels whose 2-sigma ensemble bound exceeds 2%) is
compared with the plain tracer's image of the same point: it must be faster,
and its intensities, judged by the exact tracer on a random pixel subset,
must be close; pixels sent to the fallback must carry the exact values."""
from __future__ import annotations

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_surrogate_is_faster_than_the_tracer_at_small_error(hb, gpu_ctx, sigma_table):
    import torch
    from hadros_b200 import scan
    from hadros_b200 import surrogate as S
    from hadros_b200 import workloads as W
    torch.cuda.set_device(0)
    side, bins = 512, 16
    train = [scan.production_cam(r, t, side, bins) for r, t in W.scan_points(48, seed=101)]
    raw, y, info = S.trace_samples(gpu_ctx, sigma_table, train, 4096, seed=5)
    sur = S.Surrogate(members=2, seed=3)
    sur.fit(raw, y, epochs=80, batch=8192, lr=2e-3, floors=(S.TAU_FLOOR, info["i_floor"]))
    (r0, t0), = W.scan_points(1, seed=202)
    p = scan.production_cam(r0, t0, side, bins)

    # the method without the network: the exact tracer on every pixel
    torch.cuda.synchronize()
    a = time.perf_counter()
    exact = gpu_ctx.image(p, sigma_table, outputs=("tau", "P_surv", "I_obs"))
    t_plain = time.perf_counter() - a

    # with it: surrogate image + exact fallback (warm the kernel once first)
    sur.image(p, sigma_table, threshold=0.01, per_bin=False)
    torch.cuda.synchronize()
    a = time.perf_counter()
    img = sur.image_with_fallback(gpu_ctx, p, sigma_table, threshold=0.01)
    t_sur = time.perf_counter() - a

    P = side * side
    fb = img["fallback"]
    np.testing.assert_array_equal(img["I_obs"][fb], exact["I_obs"][fb])
    judge = np.random.default_rng(7).choice(P, size=P // 100, replace=False)
    e = scan.errors(exact["I_obs"][judge], img["I_obs"][judge])
    print(f"plain {t_plain:.3f} s, surrogate {t_sur:.3f} s ({t_plain / t_sur:.1f}x), "
          f"fallback {fb.size / P:.4f}, judged error median {e['median']:.4f} worst {e['worst']:.4f}")
    assert e["n"] > 100
    assert t_sur < t_plain / 1.5
    assert fb.size < P // 2
    assert e["median"] < 0.02 and e["worst"] < 0.15
