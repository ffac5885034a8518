"""Generates the golden fixtures in tests/golden/*.npz from the REFERENCE itself.

Each case runs the reference's own code (KerrCamera::trace_pixel +
radiative_transfer::integrate_kerr_ray_spectral, built from the reference
sources by oracle/build_ref.sh into oracle/_ref/libhadros_ref.so) and stores
its per-pixel outputs together with the parameters.  Run it where the
reference sources are available:

    oracle/build_ref.sh && python tests/golden/make_golden.py [name-prefix]

The fixtures pin the CPU oracle (tests/test_oracle.py) and are what the GPU
parity tests compare against on machines without the reference.  A fixture
of a pixel subset stores the ids as `pixel_ids` (outputs in list order).
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

import hadros_b200 as hb  # noqa: E402
from hadros_b200 import workloads as W  # noqa: E402
from oracle import pyoracle as O  # noqa: E402


def cases() -> dict[str, dict]:
    c: dict[str, dict] = {}
    # The 32x32 plain tracer, whole image.
    c["plain_tracer_32"] = W.plain_tracer_32()
    # The 512x512 mixed-precision configuration, sampled at 16x16 (same
    # camera, coarser pixel grid), FP64 arithmetic.
    c["mixed_cfg_16_fp64"] = W.mixed_512(nx=16, ny=16, precision="fp64")
    # every density profile x every source morphology, 4x4, 4 cutoff bins
    for prof in hb.PROFILES:
        for src in hb.SOURCES:
            c[f"matrix_{prof}_{src}"] = W.mixed_512(nx=4, ny=4, precision="fp64", profile=prof,
                                                    source=src, h=0.05, n_bins=4)
    # spectral models
    c["spectral_powerlaw"] = W.mixed_512(nx=6, ny=6, precision="fp64", spectral="powerlaw",
                                         h=0.05, n_bins=5)
    c["spectral_mono_jet"] = W.mixed_512(nx=6, ny=6, precision="fp64", spectral="monochromatic",
                                         source="jet_base", Enu_obs_GeV=3.0e7, h=0.05)
    # edge cases
    c["edge_one_pixel"] = W.plain_tracer_32(nx=1, ny=1)
    c["edge_ragged_3x5"] = W.mixed_512(nx=3, ny=5, precision="fp64", h=0.05)
    c["edge_step_cap_40"] = W.mixed_512(nx=4, ny=4, precision="fp64", max_steps=40)
    c["edge_cap_11"] = W.mixed_512(nx=3, ny=3, precision="fp64", max_steps=11)
    c["edge_one_bin"] = W.mixed_512(nx=4, ny=4, precision="fp64", n_bins=1, h=0.05)
    c["edge_empty_band"] = W.mixed_512(nx=3, ny=3, precision="fp64", spec_e_min_GeV=1.0e13,
                                       spec_e_max_GeV=1.0e14, h=0.05)
    c["edge_energy_below_table"] = W.plain_tracer_32(nx=4, ny=4, Enu_obs_GeV=1.0e3, fov_deg=25.0,
                                                     r_obs_rg=60.0, r_max_rg=120.0, h=0.05)
    c["edge_schwarzschild"] = W.mixed_512(nx=4, ny=4, precision="fp64", a_spin=0.0, h=0.05)
    c["edge_zero_floor_gauss"] = W.plain_tracer_32(nx=4, ny=4, rho_floor_gcm3=0.0, r_obs_rg=60.0, fov_deg=25.0,
                                                   r_max_rg=120.0, h=0.05)
    c["edge_source_guard"] = W.mixed_512(nx=3, ny=3, precision="fp64", source="inner_ring",
                                         src_sigma_r_rg=0.0, h=0.05)
    c["edge_equatorial_wide"] = W.mixed_512(nx=5, ny=5, precision="fp64", theta_obs_deg=89.0,
                                            fov_deg=60.0, h=0.05, a_spin=0.7)
    c["edge_polar"] = W.mixed_512(nx=3, ny=3, precision="fp64", theta_obs_deg=2.0, h=0.05)
    # MeV thermal channel (mev_* fixtures also store its five outputs)
    col = dict(nx=5, ny=4, h=0.05, a_spin=0.95, theta_obs_deg=70.0, r_obs_rg=60.0, r_max_rg=120.0,
               fov_deg=25.0, M_bh_msun=3.0, rho0_gcm3=1.0e11, profile="collapsar_ndaf_like", r0_rg=12.0,
               sigma_r_rg=8.0, H_over_R=0.45, torus_r_min_rg=3.0, torus_r_max_rg=80.0,
               rho_floor_gcm3=1.0e-3, source="density_weighted", precision="fp64", mev_channel=1)
    c["mev_physical_collapsar"] = dict(col)
    for th, ye in zip(("constant", "inner_hot_torus", "radial_powerlaw", "torus_plus_cool_envelope",
                       "collapsar_inner_hot"),
                      ("collapsar_neutron_rich", "constant", "neutron_rich_torus", "funnel_proton_rich",
                       "torus_envelope_contrast")):
        c[f"mev_T_{th}"] = dict(col, nx=4, ny=4, mev_thermal=th, mev_ye=ye)
    c["mev_nu_e_degeneracy"] = dict(col, nx=4, ny=3, mev_flavor="nu_e", mev_degeneracy_correction=True)
    c["mev_nu_x"] = dict(col, nx=4, ny=3, mev_flavor="nu_x", mev_Enu_obs_MeV=25.0)
    c["mev_toy"] = dict(col, nx=4, ny=3, mev_model="toy", mev_norm=1.0e-40)
    c["mev_fd_band_spectral"] = dict(col, nx=4, ny=3, mev_spectral="fermi_dirac_band", mev_n_bins=5,
                                     spectral="powerlaw_cutoff", n_bins=4)
    c["mev_empty_band"] = dict(col, nx=3, ny=3, spectral="powerlaw", spec_e_min_GeV=1.0e13,
                               spec_e_max_GeV=1.0e14)
    c["mev_switches_off"] = dict(col, nx=4, ny=3, mev_pair=False, mev_scat_e=False, mev_abs_p=False,
                                 mev_neutrinosphere_tau=5.0)
    c["mev_gaussian_thin"] = W.mixed_512(nx=4, ny=4, precision="fp64", h=0.05, mev_channel=1,
                                         rho0_gcm3=1.0e8, mev_thermal="radial_powerlaw")
    # The production-scan camera at its own settings (4096x4096, h0 0.01, 64
    # bins): an 8x8 strided pixel sample (every 512th pixel in i and j, from
    # 256), at a mid-box point and at a dense, nearly face-on one.
    side = 4096
    ii = 256 + 512 * np.arange(8)
    ids = (ii[:, None] * side + ii[None, :]).ravel().astype(np.int32)
    c["production_c5_mid_8x8"] = dict(W.production_point(precision="fp64"), _pixel_ids=ids)
    c["production_c5_dense_8x8"] = dict(W.production_point(precision="fp64", rho0_gcm3=1.0e12,
                                                           theta_obs_deg=15.0), _pixel_ids=ids)
    # The pixels of the 512x512 camera traced at 256x256 whose accepted-step
    # count came out one off the reference in a full-image comparison on the
    # GPU (65,536 rays): rays with a near-tie accept/reject decision.
    c["scale_c2_256_near_ties"] = dict(W.mixed_512(nx=256, ny=256, precision="fp64"),
                                       _pixel_ids=np.array([27795, 31311, 34200, 34658, 38802, 39770, 42099],
                                                           dtype=np.int32))
    return c


def main() -> None:
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libhadros_ref.so missing: run oracle/build_ref.sh first")
    E, g2, s = W.synthetic_sigma_arrays()
    np.savez(HERE / "sigma_synthetic.npz", E=E, sigma_GeV2=g2, sigma_cm2=s)
    only = sys.argv[1] if len(sys.argv) > 1 else ""   # optional name prefix
    for name, kw in cases().items():
        if not name.startswith(only):
            continue
        kw = dict(kw)
        ids = kw.pop("_pixel_ids", None)   # a pixel subset, stored as pixel_ids
        p = hb.params(**kw)
        out = O.ref_image(p, E, g2, s, pixel_ids=ids, mev=name.startswith("mev_"))
        if ids is not None:
            out["pixel_ids"] = ids
        meta = {k: (v if not isinstance(v, (np.floating, np.integer)) else v.item())
                for k, v in kw.items()}
        np.savez_compressed(HERE / f"{name}.npz", params=json.dumps(meta), **out)
        print(f"{name}: steps {out['steps'].min()}..{out['steps'].max()} "
              f"fates {np.bincount(out['fate'], minlength=3).tolist()}", flush=True)


if __name__ == "__main__":
    main()
