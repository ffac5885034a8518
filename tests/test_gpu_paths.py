"""Geodesic cache on the GPU: recorded paths against the oracle's, and the
transfer over cached paths against the fused image and the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from parity import RTOL_FP64, RTOL_MIXED, assert_parity

pytestmark = pytest.mark.gpu


def test_trace_paths_match_oracle(hb, gpu_ctx, sigma_arrays):
    from hadros_b200 import workloads as W
    from test_kgeo import oracle_paths
    E, _, s = sigma_arrays
    p = hb.params(**W.mixed_512(nx=4, ny=3, h=0.05, precision="fp64"))
    got = gpu_ctx.trace_paths(p, max_points=8000)
    n, pts, fate = oracle_paths(hb, p, E, s)
    np.testing.assert_array_equal(got["npoints"], n)
    np.testing.assert_array_equal(got["fate"], fate)
    mine = hb.pack_paths(got["points"], got["npoints"])
    # ulp-level differences (CUDA vs glibc libm) grow where the redshift
    # diverges, on the last steps of captured rays: most points agree to 1e-6,
    # all to 1e-3
    rel = np.abs(mine - pts) / np.maximum(np.abs(pts), 1e-9)
    assert np.mean(rel[:, [0, 1, 5, 6]] > 1e-6) < 0.01
    assert np.max(rel[:, [0, 1, 5, 6]]) < 1e-3
    assert np.max(np.abs(mine[:, 2:5] - pts[:, 2:5])) < 1e-3


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_transfer_over_own_paths_equals_fused_image(hb, gpu_ctx, sigma_table, precision):
    from hadros_b200 import workloads as W
    p = hb.params(**W.mixed_512(nx=5, ny=4, h=0.05, precision=precision))
    fused = gpu_ctx.image(p, sigma_table)
    paths = gpu_ctx.trace_paths(p, max_points=8000)
    img = gpu_ctx.transfer_paths(p, sigma_table, paths["npoints"],
                                 hb.pack_paths(paths["points"], paths["npoints"]), paths["fate"])
    for k in ("tau", "P_surv", "I_obs", "fate", "steps", "tau_E", "I_E"):
        np.testing.assert_array_equal(img[k], fused[k], err_msg=k)


@pytest.mark.parametrize("precision,rtol", [("fp64", RTOL_FP64), ("mixed", RTOL_MIXED)])
def test_transfer_over_cpu_cache_matches_oracle(hb, gpu_ctx, sigma_table, sigma_arrays, tmp_path,
                                                precision, rtol):
    """A cache made on the CPU (oracle paths, written and read as KGEO) and
    transferred on the GPU: the reference's two-process flow."""
    from hadros_b200 import workloads as W
    from oracle import pyoracle as O
    from test_kgeo import oracle_paths
    E, _, s = sigma_arrays
    kw = W.mixed_512(nx=4, ny=4, h=0.05, precision=precision, source="inner_ring",
                     profile="gaussian", rho0_gcm3=1e9)
    p = hb.params(**kw)
    n, pts, fate = oracle_paths(hb, p, E, s)
    hb.write_kgeo(tmp_path / "c.bin", p, n, pts, fate=fate)
    d = hb.read_kgeo(tmp_path / "c.bin")
    img = gpu_ctx.transfer_paths(p, sigma_table, d["npoints"], d["points"],
                                 np.where(d["captured"] == 1, 1, 0).astype(np.int8))
    ref = O.oracle_image(p, E, s)
    ref["fate"] = (ref["fate"] == 1).astype(np.int8)   # KGEO keeps only `captured`
    assert_parity(img, ref, rtol, f"cache/{precision}", p_absolute=(precision == "mixed"))


def test_transfer_paths_energy_scan_reuses_geometry(hb, gpu_ctx, sigma_table):
    """One traced geometry, many energies: each equals a fresh image."""
    from hadros_b200 import workloads as W
    p = hb.params(**W.plain_tracer_32(nx=4, ny=4, r_obs_rg=60.0, r_max_rg=120.0, fov_deg=25.0,
                                      h=0.05))
    paths = gpu_ctx.trace_paths(p, max_points=6000)
    packed = hb.pack_paths(paths["points"], paths["npoints"])
    for E in (1e5, 1e7, 1e11):
        q = p.copy()
        q.Enu_obs_GeV = E
        a = gpu_ctx.transfer_paths(q, sigma_table, paths["npoints"], packed, paths["fate"])
        b = gpu_ctx.image(q, sigma_table)
        np.testing.assert_array_equal(a["tau"], b["tau"])
        np.testing.assert_array_equal(a["I_obs"], b["I_obs"])
