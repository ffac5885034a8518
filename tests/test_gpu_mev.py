"""The MeV thermal channel on the GPU (radiative_transfer.cpp:522-638 with
mev_neutrino_physics.cpp): against the CPU oracle live on random settings,
bit for bit across the library's launch paths (single image, batch of
cameras with the channel on and off, plan, deferred transfer, cached paths,
no-alloc entry point), and without effect on the UHE outputs.  The golden
fixtures mev_* run through every precision in test_gpu_parity.py.  Needs a
B200."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from parity import MEV_KEYS, RTOL_FP64, RTOL_MIXED, assert_parity, mev_errors

pytestmark = pytest.mark.gpu

UHE_KEYS = ("tau", "P_surv", "I_obs", "fate", "steps", "attempts", "tau_E", "I_E")


def _collapsar(**over) -> dict:
    d = dict(nx=5, ny=4, h=0.05, a_spin=0.95, theta_obs_deg=70.0, r_obs_rg=60.0, r_max_rg=120.0, fov_deg=25.0,
             rho0_gcm3=1.0e11, profile="collapsar_ndaf_like", r0_rg=12.0, sigma_r_rg=8.0, H_over_R=0.45,
             torus_r_min_rg=3.0, torus_r_max_rg=80.0, rho_floor_gcm3=1.0e-3, source="density_weighted",
             spectral="powerlaw_cutoff", n_bins=6, precision="fp64", fast=False, mev_channel=1)
    d.update(over)
    return d


def test_random_settings_vs_live_oracle(hb, gpu_ctx, sigma_table, sigma_arrays):
    from hadros_b200 import workloads as W
    from oracle import pyoracle as O
    E, _, s = sigma_arrays
    rng = np.random.default_rng(77)
    names = dict(mev_thermal=["constant", "inner_hot_torus", "radial_powerlaw", "torus_plus_cool_envelope",
                              "collapsar_inner_hot"],
                 mev_ye=["constant", "neutron_rich_torus", "funnel_proton_rich", "torus_envelope_contrast",
                         "collapsar_neutron_rich"],
                 mev_flavor=["nu_e", "anti_nu_e", "nu_x"], mev_model=["toy", "physical"],
                 mev_spectral=["monochromatic", "fermi_dirac_band"])
    for k in range(6):
        kw = W.mixed_512(nx=int(rng.integers(2, 6)), ny=int(rng.integers(2, 6)), h=float(rng.uniform(0.03, 0.08)),
                         a_spin=float(rng.uniform(0.0, 0.998)), theta_obs_deg=float(rng.uniform(10.0, 85.0)),
                         profile=int(rng.integers(0, 8)), source=int(rng.integers(0, 5)),
                         spectral=int(rng.integers(0, 3)), n_bins=int(rng.integers(1, 9)),
                         rho0_gcm3=float(10.0 ** rng.uniform(8, 12)), precision="fp64", mev_channel=1,
                         mev_n_bins=int(rng.integers(1, 9)), mev_T0_MeV=float(rng.uniform(2.0, 12.0)),
                         mev_degeneracy_correction=bool(rng.integers(0, 2)),
                         mev_scattering=bool(rng.integers(0, 2)),
                         **{key: str(rng.choice(v)) for key, v in names.items()})
        p = hb.params(**kw)
        ref = O.oracle_image(p, E, s, mev=True)
        for fast in (False, True):
            p.fast_geodesic = int(fast)
            p.precision = hb.PRECISION_FP64
            assert_parity(gpu_ctx.image(p, sigma_table), ref, RTOL_FP64, f"random {k} fast={fast}/fp64")
            p.precision = hb.PRECISION_MIXED
            assert_parity(gpu_ctx.image(p, sigma_table), ref, RTOL_MIXED, f"random {k} fast={fast}/mixed",
                          p_absolute=True)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_channel_leaves_uhe_outputs_alone(hb, gpu_ctx, sigma_table, precision):
    """Switching the channel on adds its outputs and changes no other bit;
    switched off, requested MeV outputs hold RTResult's defaults."""
    on = hb.params(**_collapsar(precision=precision))
    off = hb.params(**_collapsar(precision=precision, mev_channel=0))
    a = gpu_ctx.image(on, sigma_table)
    b = gpu_ctx.image(off, sigma_table, outputs=hb.OUTPUTS + hb.MEV_OUTPUTS)
    for k in UHE_KEYS:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for k, v in zip(MEV_KEYS, (0.0, 1.0, 0.0, -1.0, 1.0)):
        np.testing.assert_array_equal(b[k], v, err_msg=k)
    assert a["tau_mev"].max() > 0.0 and (a["I_obs_mev"] > 0.0).all()


def test_batch_and_plan_with_channel_on_some_cameras(hb, gpu_ctx, sigma_table):
    """One launch over cameras with and without the channel gives each
    camera its own image's outputs, bit for bit."""
    import torch
    cams = [hb.params(**_collapsar(nx=4, ny=3)),
            hb.params(**_collapsar(nx=3, ny=5, mev_channel=0, theta_obs_deg=40.0)),
            hb.params(**_collapsar(nx=2, ny=4, mev_thermal="radial_powerlaw", mev_flavor="nu_e",
                                   mev_spectral="fermi_dirac_band", a_spin=0.5))]
    singles = [gpu_ctx.image(c, sigma_table, outputs=hb.OUTPUTS + hb.MEV_OUTPUTS) for c in cams]
    batch = gpu_ctx.batch(cams, sigma_table)
    for k, (got, ref) in enumerate(zip(batch, singles)):
        for key in UHE_KEYS + MEV_KEYS:
            np.testing.assert_array_equal(got[key], ref[key], err_msg=f"batch camera {k} {key}")
    plan = gpu_ctx.plan(cams, sigma_table, hb.schedule(order=hb.ORDER_TILES))
    out = plan.alloc(torch, device=torch.device("cuda", 0))
    assert all(k in out for k in MEV_KEYS)
    plan.launch(out, torch.cuda.current_stream())
    torch.cuda.synchronize()
    got = {k: v.cpu().numpy() for k, v in out.items()}
    o = 0
    for k, ref in enumerate(singles):
        P = cams[k].nx * cams[k].ny
        for key in MEV_KEYS:
            np.testing.assert_array_equal(got[key][o:o + P], ref[key], err_msg=f"plan camera {k} {key}")
        o += P
    plan.close()


def test_deferred_transfer_keeps_the_channel(hb, gpu_ctx, sigma_table):
    """Many bins (deferred transfer) and few (in the loop): the same MeV bits."""
    p = hb.params(**_collapsar(precision="mixed", n_bins=32))
    gpu_ctx.set_transfer("deferred")
    a = gpu_ctx.image(p, sigma_table)
    gpu_ctx.set_transfer("in_loop")
    b = gpu_ctx.image(p, sigma_table)
    gpu_ctx.set_transfer("auto")
    for k in UHE_KEYS + MEV_KEYS:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cached_paths_give_the_fused_channel(hb, gpu_ctx, sigma_table, precision):
    """compute_kerr_image_from_cache computes the MeV columns from the cache:
    the cached-path kernel gives the fused kernel's values bit for bit."""
    p = hb.params(**_collapsar(precision=precision))
    fused = gpu_ctx.image(p, sigma_table)
    paths = gpu_ctx.trace_paths(p, max_points=8000)
    img = gpu_ctx.transfer_paths(p, sigma_table, paths["npoints"],
                                 hb.pack_paths(paths["points"], paths["npoints"]), paths["fate"])
    for k in ("tau", "P_surv", "I_obs", "tau_E", "I_E") + MEV_KEYS:
        np.testing.assert_array_equal(img[k], fused[k], err_msg=k)


def test_noalloc_entry_point_computes_the_channel(hb, gpu_ctx, sigma_table):
    import torch
    torch.cuda.set_device(0)
    p = hb.params(**_collapsar(nx=4, ny=4))
    ref = gpu_ctx.image(p, sigma_table)
    dev = torch.device("cuda", 0)
    bufs = {k: torch.full((16,), -7.0, dtype=torch.float64, device=dev) for k in MEV_KEYS}
    bufs["steps"] = torch.full((16,), -1, dtype=torch.int32, device=dev)
    out = hb.HadrosImageOut()
    for k, t in bufs.items():
        setattr(out, k, t.data_ptr())
    torch.cuda.synchronize()
    rc = hb.lib().hadros_image_device_noalloc(C.byref(p), sigma_table.handle, C.byref(out),
                                               C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, hb.lib().hadros_last_error().decode()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(bufs["steps"].cpu().numpy(), ref["steps"])
    for k in MEV_KEYS:   # the same kernel source built in another translation unit
        np.testing.assert_allclose(bufs[k].cpu().numpy(), ref[k], rtol=1e-12, atol=0.0, err_msg=k)


def test_mev_fixture_errors_are_tiny(hb, gpu_ctx, sigma_table):
    """Reference-arithmetic FP64 kernel on the thick collapsar fixture: the
    channel agrees with the reference to libm rounding, far inside 1e-6."""
    from conftest import load_golden
    kw, ref = load_golden("mev_physical_collapsar")
    got = gpu_ctx.image(hb.params(**dict(kw, precision="fp64", fast=False)), sigma_table)
    errs = mev_errors(got, ref)
    assert max(errs.values()) < 1e-9, errs
