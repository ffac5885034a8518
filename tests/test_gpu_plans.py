"""Plans: scans uploaded once, launched on a stream (and replayed from a CUDA
graph), under every schedule the autotuner can pick; outputs must not depend
on the schedule."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cams(hb, n=5, seed=3):
    from hadros_b200 import workloads as W
    rng = np.random.default_rng(seed)
    return [hb.params(**W.mixed_512(nx=int(rng.integers(3, 20)), ny=int(rng.integers(3, 20)), h=0.05,
                                    a_spin=float(rng.uniform(0, 0.998)),
                                    theta_obs_deg=float(rng.uniform(5, 85)), profile=k % 8,
                                    n_bins=int(rng.integers(1, 10)), precision="mixed"))
            for k in range(n)]


def _host(out):
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize("order", [0, 1, 2])
@pytest.mark.parametrize("bps", [0, 2])
def test_plan_equals_batch_under_every_schedule(hb, gpu_ctx, sigma_table, order, bps):
    import torch
    cams = _cams(hb)
    ref = gpu_ctx.batch(cams, sigma_table)
    plan = gpu_ctx.plan(cams, sigma_table, hb.schedule(order=order, blocks_per_sm=bps, coarse_stride=4))
    out = plan.alloc(torch, device=torch.device("cuda", 0))
    plan.launch(out, torch.cuda.current_stream())
    c = plan.counters(torch.cuda.current_stream())
    got = _host(out)
    o = ob = 0
    for k, cam in enumerate(cams):
        P, B = cam.nx * cam.ny, hb.n_bins_of(cam)
        for key in ref[k]:
            g = got[key][ob:ob + P * B].reshape(P, B) if key in ("tau_E", "I_E") else got[key][o:o + P]
            np.testing.assert_array_equal(g, ref[k][key], err_msg=f"camera {k} {key}")
        o += P
        ob += P * B
    assert c["accepted_steps"] == int(got["steps"].astype(np.int64).sum())
    plan.close()


def test_plan_replays_from_cuda_graph(hb, gpu_ctx, sigma_table):
    import torch
    cams = _cams(hb, n=3, seed=8)
    plan = gpu_ctx.plan(cams, sigma_table)
    out = plan.alloc(torch, device=torch.device("cuda", 0))
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        plan.launch(out, s)                     # eager reference
    torch.cuda.synchronize()
    ref = _host(out)
    for t in out.values():
        t.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        plan.launch(out, s)
    for _ in range(2):
        for t in out.values():
            t.zero_()
        g.replay()
        torch.cuda.synchronize()
        got = _host(out)
        for k in ref:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    del g
    plan.close()


def test_autotuner_picks_and_caches(hb, gpu_ctx, sigma_table, tmp_path, monkeypatch):
    import torch
    from hadros_b200 import autotune
    monkeypatch.setenv("HADROS_B200_CACHE", str(tmp_path / "tune.json"))
    cams = _cams(hb, n=3, seed=9)
    best, rep = autotune.autotune(gpu_ctx, cams, sigma_table, torch, scale=1, repeats=1)
    assert not rep["cached"] and len(rep["timings"]) == len(autotune.CANDIDATES)
    best2, rep2 = autotune.autotune(gpu_ctx, cams, sigma_table, torch, scale=1, repeats=1)
    assert rep2["cached"] and bytes(best2) == bytes(best)


def test_batch_pixels_equals_per_camera_pixel_lists(hb, gpu_ctx, sigma_table):
    """hadros_batch_pixels (pixel subsets of several cameras in one launch)
    gives, per camera, exactly what hadros_image_pixels gives for its list."""
    from hadros_b200 import workloads as W
    rng = np.random.default_rng(11)
    cams = [hb.params(**W.mixed_512(nx=48, ny=40, h=0.05, theta_obs_deg=t, rho0_gcm3=r))
            for t, r in ((17.0, 1e11), (45.0, 1e9), (70.0, 3e10))]
    lists = [np.sort(rng.choice(48 * 40, size=n, replace=False)).astype(np.int32) for n in (37, 0, 150)]
    got = gpu_ctx.batch_pixels(cams, sigma_table, lists)
    for p, ids, g in zip(cams, lists, got):
        if ids.size == 0:
            assert all(v.size == 0 for v in g.values())
            continue
        ref = gpu_ctx.image(p, sigma_table, pixel_ids=ids)
        for k in ref:
            np.testing.assert_array_equal(g[k], ref[k], err_msg=k)
    with pytest.raises(hb.HadrosError):
        gpu_ctx.batch_pixels(cams[:1], sigma_table, [np.array([48 * 40], dtype=np.int32)])
