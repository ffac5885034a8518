"""Host-side logic of the surrogate scans (hadros_b200/scan.py): the judged
error metric and the scan workloads' parameter boxes."""
from __future__ import annotations

import math

import numpy as np

from hadros_b200 import scan
from hadros_b200 import workloads as W


def test_errors_counts_only_pixels_above_the_floor():
    ex = np.array([1.0, 0.5, 1e-7, 0.0, 2.0])
    sur = np.array([1.01, 0.45, 5e-7, 3.0, 2.0])
    e = scan.errors(ex, sur, floor_rel=1e-6)
    # the 1e-7 and 0 pixels are below 1e-6 * 2.0 and are not judged
    assert e["n"] == 3
    assert math.isclose(e["worst"], 0.1)
    assert math.isclose(e["median"], 0.01)


def test_errors_of_an_all_dark_image():
    e = scan.errors(np.zeros(10), np.ones(10))
    assert e == {"n": 0, "worst": 0.0, "p99": 0.0, "median": 0.0}


def test_scan_points_cover_the_production_box():
    pts = W.scan_points(256)
    rho = np.array([r for r, _ in pts])
    th = np.array([t for _, t in pts])
    assert len(pts) == 256
    assert rho.min() >= 1e9 and rho.max() <= 1e12
    assert th.min() >= 10.0 and th.max() <= 80.0
    assert np.log10(rho).std() > 0.7          # log-uniform over three decades
    assert W.scan_points(256) == pts           # seeded


def test_training_cameras_are_seeded_and_vary_what_config_4_varies():
    cams = W.surrogate_training_cams(64)
    assert cams == W.surrogate_training_cams(64)
    prof = {c["profile"] for c in cams}
    assert len(prof) == 8
    a = np.array([c["a_spin"] for c in cams])
    assert a.min() >= 0.0 and a.max() <= 0.998
    cos_i = np.cos(np.radians([c["theta_obs_deg"] for c in cams]))
    assert cos_i.min() >= math.cos(math.radians(85.0)) - 1e-12
    assert all(c["envelope_rho0_gcm3"] == 0.01 * c["rho0_gcm3"] for c in cams)


def test_calibration_picks_the_largest_safe_threshold(hb, sigma_table):
    """calibrate(): the threshold is the largest spread below which held-out
    pixels rarely err beyond the bound.  A stand-in ensemble whose pixels have
    spread d_i and error 0.5% below spread 0.004 but 3% above it must get a
    threshold just below 0.004 when no bad pixel may pass (q = 0.999), and
    at most two steps of the threshold grid (5.8% each) above it with the
    default q = 0.99, which admits a 1% tail for the scan's escalation."""
    import torch

    B, P, K = 4, 2000, 4
    p = hb.params(**W.production_point(nx=64, ny=64, n_bins=B))
    rng = np.random.default_rng(3)
    lnI_true = rng.uniform(-70, -50, size=(P, B))
    floor = 1e-40
    y = np.stack([np.zeros(P * B), np.log(np.exp(lnI_true).reshape(-1) + floor)], axis=1)
    d = np.geomspace(2e-4, 1e-2, P)
    e = np.where(d < 0.004, 0.005, 0.03)
    offs = np.array([1.0, -1.0, 1.0, -1.0])[:, None, None] * d[None, :, None]
    lnI_k = lnI_true[None] + np.log1p(e)[None, :, None] + offs

    class Ens:
        def forward(self, raw):
            out = np.zeros((K, P * B, 2))
            out[:, :, 1] = lnI_k.reshape(K, -1)
            return torch.from_numpy(out)

    raw = torch.zeros((P * B, 16))
    c = scan.calibrate(Ens(), sigma_table, [p], raw, torch.from_numpy(y), floor, bound=0.01, q=0.999)
    assert c["pixels"] > 0.5 * P
    assert 0.0025 < c["threshold"] < 0.004
    assert abs(c["fallback_frac_held_out"] - (d > c["threshold"]).mean()) < 0.02
    c = scan.calibrate(Ens(), sigma_table, [p], raw, torch.from_numpy(y), floor, bound=0.01)
    assert 0.0025 < c["threshold"] < 0.004 * 1.0583 ** 2
