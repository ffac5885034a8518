"""The scan point's device path (hadros_b200.scan.PointRunner) and the
device pixel-list entry point under it (hadros_image_pixels_device), through
the C ABI.

* A device id list traces the same rays, bit for bit, as the host list of
  hadros_image_pixels.
* With a threshold below every spread, every pixel falls back: the finished
  image must then equal the plain tracer's image exactly, and the judged
  error must be zero.  This holds whatever the network predicts, so the
  networks here are untrained.
* The host-to-host form (run_host) returns the same image as run()."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("tau", "P_surv", "I_obs")


def _cam(hb, side=16, bins=8):
    from hadros_b200 import workloads as W
    return hb.params(**W.production_point(nx=side, ny=side, n_bins=bins, h=0.05, rho0_gcm3=3e10,
                                          theta_obs_deg=40.0))


def _untrained(hb, members=2):
    from hadros_b200 import surrogate as S
    sur = S.Surrogate(members=members, device=0, seed=3)
    nm = hb.abi.HadrosMlpNorm()
    mu = [0.0, 0.0, 0.9, 0.5, 10.5] + [0.0] * 8 + [10.0, 0.3, 8.0]
    sd = [7.7, 7.7, 0.3, 0.3, 1.0] + [1.0] * 8 + [2.3, 0.1, 2.0]
    for j in range(16):
        nm.feat_mu[j], nm.feat_inv_sd[j] = mu[j], 1.0 / sd[j]
    nm.out_mu[0], nm.out_sd[0], nm.out_mu[1], nm.out_sd[1] = 5.0, 6.0, -60.0, 8.0
    nm.out_floor[0] = S.TAU_FLOOR
    sur.norm = nm
    return sur


def test_device_pixel_list_equals_host_pixel_list(hb, gpu_ctx, sigma_table):
    import torch
    torch.cuda.set_device(0)
    p = _cam(hb)
    ids = np.random.default_rng(11).choice(256, size=57, replace=False).astype(np.int32)
    ref = gpu_ctx.image(p, sigma_table, pixel_ids=ids, outputs=KEYS + ("fate", "steps"))
    dev = torch.device("cuda", 0)
    out = {k: torch.full((ids.size,), -7.0, dtype=torch.float64, device=dev) for k in KEYS}
    out["fate"] = torch.full((ids.size,), -1, dtype=torch.int8, device=dev)
    out["steps"] = torch.full((ids.size,), -1, dtype=torch.int32, device=dev)
    t_ids = torch.from_numpy(ids).to(dev)
    gpu_ctx.pixels_device(p, sigma_table, t_ids, out)
    torch.cuda.synchronize()
    for k in KEYS + ("fate", "steps"):
        np.testing.assert_array_equal(out[k].cpu().numpy(), ref[k], err_msg=k)
    # the first n ids only
    part = {k: v[:20].clone().fill_(-7) for k, v in out.items()}
    gpu_ctx.pixels_device(p, sigma_table, t_ids, part, n=20)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(part["steps"].cpu().numpy(), ref["steps"][:20])


def test_point_runner_with_every_pixel_falling_back_is_the_plain_image(hb, gpu_ctx, sigma_table):
    import torch
    from hadros_b200 import scan as SC
    torch.cuda.set_device(0)
    p = _cam(hb)
    sur = _untrained(hb)
    runner = SC.PointRunner(gpu_ctx, sigma_table, sur, 16, 8, judge_frac=0.1)
    jids = SC.judge_ids(256, 0.1, np.random.default_rng(5))
    res = runner.run(p, -1.0, jids)
    plain = gpu_ctx.image(p, sigma_table, outputs=KEYS)
    assert res["fallback_pixels"] == 256 and res["judged"] == jids.size
    for k in KEYS:
        np.testing.assert_array_equal(runner.out[k].cpu().numpy(), plain[k], err_msg=k)
    assert res["error"]["worst"] == 0.0 and res["P_surv_max_abs_error"] == 0.0
    # host to host: the same image
    host = runner.alloc_host()
    host["judge_ids"].copy_(torch.from_numpy(jids))
    r2 = runner.run_host(p, -1.0, host)
    assert r2["fallback_pixels"] == 256, r2
    assert r2["d2h_bytes"] >= 3 * 8 * 256 and r2["h2d_bytes"] >= 4 * jids.size
    for k in KEYS:
        np.testing.assert_array_equal(runner.out[k].cpu().numpy(), plain[k], err_msg=f"device {k}")
        np.testing.assert_array_equal(host[k].numpy(), plain[k], err_msg=f"host {k}")


def test_point_runner_judges_the_surrogate_where_nothing_falls_back(hb, gpu_ctx, sigma_table):
    """With no fallback the judged error is the surrogate's own, measured
    against the exact tracer on the judge pixels."""
    import torch
    from hadros_b200 import scan as SC
    torch.cuda.set_device(0)
    p = _cam(hb)
    sur = _untrained(hb)
    runner = SC.PointRunner(gpu_ctx, sigma_table, sur, 16, 8, judge_frac=0.25)
    jids = SC.judge_ids(256, 0.25, np.random.default_rng(6))
    res = runner.run(p, 1e30, jids, detail=True)
    assert res["fallback_pixels"] == 0
    ex = gpu_ctx.image(p, sigma_table, pixel_ids=jids, outputs=KEYS)
    np.testing.assert_array_equal(res["judge"]["exact"]["I_obs"], ex["I_obs"])
    want = SC.errors(ex["I_obs"], runner.out["I_obs"].cpu().numpy()[jids])
    assert res["error"]["n"] == want["n"]
    assert res["error"]["worst"] == pytest.approx(want["worst"], rel=1e-12)


def test_point_runner_escalates_when_the_judge_finds_a_large_error(hb, gpu_ctx, sigma_table):
    """An untrained ensemble errs far beyond 1 %: with no pixel sent to the
    tracer by the first threshold, escalation to a threshold below every
    spread traces each pixel whose spread exceeds it, after which the image is
    the plain tracer's on those pixels and the judged error is zero."""
    import torch
    from hadros_b200 import scan as SC
    torch.cuda.set_device(0)
    p = _cam(hb)
    sur = _untrained(hb)
    runner = SC.PointRunner(gpu_ctx, sigma_table, sur, 16, 8, judge_frac=0.25)
    jids = SC.judge_ids(256, 0.25, np.random.default_rng(8))
    base = runner.run(p, 1e30, jids)
    assert base["fallback_pixels"] == 0 and base["error"]["worst"] > 0.01
    res = runner.run(p, 1e30, jids, escalate=(1e-30,), bound=0.01)
    flagged = int((runner.out["spread"] > 1e-30).sum().item())
    assert res["threshold_used"] == 1e-30 and res["escalated_pixels"] == flagged == res["fallback_pixels"]
    plain = gpu_ctx.image(p, sigma_table, outputs=KEYS)
    sp = runner.out["spread"].cpu().numpy()
    for k in KEYS:
        np.testing.assert_array_equal(runner.out[k].cpu().numpy()[sp > 1e-30], plain[k][sp > 1e-30], err_msg=k)
    if (sp > 1e-30)[jids].all():
        assert res["error"]["worst"] == 0.0
