"""Named workloads: the synthetic sigma table and the camera configurations
the pipeline is measured and checked on.

No dataset is involved: every input is synthetic and seeded.  Camera values
that a workload does not state take the reference Makefile defaults
(CAM_R_OBS_RG 60, CAM_FOV_DEG 25, CAM_R_MAX_RG 120, SOURCE_* values,
Makefile:49-153), the small-validation step h0 = 0.01 (SMALL_CAM_STEP,
Makefile:227), M = 3 Msun, the CPU tolerance 1e-6 and the 200000 step cap.
"""
from __future__ import annotations

import math

import numpy as np

SEED = 20261203


def synthetic_sigma_arrays(n: int = 81, e_lo: float = 1.0e4, e_hi: float = 1.0e12):
    """sigma_CC(E) = 7.84e-36 cm^2 (E/GeV)^0.363 at n log-spaced energies.

    Returns (E_GeV, sigma_GeV^-2, sigma_cm2); 1 GeV^-2 = 0.389379e-27 cm^2.
    """
    E = np.logspace(math.log10(e_lo), math.log10(e_hi), n)
    s_cm2 = 7.84e-36 * E ** 0.363
    s_gev2 = s_cm2 / 0.389379e-27
    return E, s_gev2, s_cm2


def write_sigma_file(path, E, s_gev2, s_cm2) -> None:
    """Write a table in the reference's 3-column format (data/sigma/*.dat);
    %.17g round-trips every double through the reference's parser."""
    with open(path, "w") as f:
        f.write("# model synthetic\n# Enu_GeV sigma_GeV_minus2 sigma_cm2\n")
        for e, g, c in zip(E, s_gev2, s_cm2):
            f.write(f"{e:.17g} {g:.17g} {c:.17g}\n")


# Makefile source defaults (Makefile:103-142).
_SOURCE_DEFAULTS = dict(src_r_center_rg=3.5, src_sigma_r_rg=1.0, src_theta_width_deg=15.0,
                        src_powerlaw=2.0, src_emax_GeV=1.0e12, src_norm=1.0,
                        src_funnel_theta_deg=20.0)


def plain_tracer_32(**over) -> dict:
    """32x32 plain tracer, FP64: a=0.9, inclination 60 deg, camera at r=1000 M
    with a 30x30 M field (fov = 2 atan(15/1000)), M=3 Msun, step cap 20000,
    gaussian torus rho0=1e10 at r0=10 with widths 3 M (sigma_r=3, H/R=0.3),
    floor 1e-3, inner_ring source, monochromatic 1e9 GeV."""
    d = dict(nx=32, ny=32, a_spin=0.9, theta_obs_deg=60.0, r_obs_rg=1000.0, r_max_rg=1000.0,
             fov_deg=2.0 * math.degrees(math.atan(15.0 / 1000.0)), h=0.1, max_steps=20000,
             M_bh_msun=3.0, profile="gaussian", rho0_gcm3=1.0e10, r0_rg=10.0, sigma_r_rg=3.0,
             H_over_R=0.3, rho_floor_gcm3=1.0e-3, source="inner_ring", spectral="monochromatic",
             Enu_obs_GeV=1.0e9, precision="fp64", **_SOURCE_DEFAULTS)
    d.update(over)
    return d


def mixed_512(**over) -> dict:
    """512x512 mixed precision: a=0.998, inclination 17 deg, powerlaw_funnel_envelope
    (rho0=1e11, index -1.5, funnel half-angle 20 deg, depletion 1, envelope 0.01 rho0,
    floor 1e-3), funnel_wall source, powerlaw_cutoff gamma=2, Ecut=1e12, 8 bins
    1e5-1e12 GeV; camera r=60, fov 25 deg, r_max 120, h0=0.01."""
    d = dict(nx=512, ny=512, a_spin=0.998, theta_obs_deg=17.0, r_obs_rg=60.0, r_max_rg=120.0,
             fov_deg=25.0, h=0.01, max_steps=200000, M_bh_msun=3.0,
             profile="powerlaw_funnel_envelope", rho0_gcm3=1.0e11, radial_power=1.5,
             funnel_theta_deg=20.0, funnel_depletion=1.0, envelope_rho0_gcm3=1.0e9,
             envelope_alpha=2.5, rho_floor_gcm3=1.0e-3, torus_r_min_rg=4.0, torus_r_max_rg=60.0,
             r0_rg=10.0, sigma_r_rg=5.0, H_over_R=0.25, source="funnel_wall",
             spectral="powerlaw_cutoff", spec_gamma=2.0, spec_ecut_GeV=1.0e12,
             spec_e_min_GeV=1.0e5, spec_e_max_GeV=1.0e12, n_bins=8, precision="mixed",
             **_SOURCE_DEFAULTS)
    d.update(over)
    return d


def batched_scan(n_cams: int = 64, seed: int = SEED, min_side: int = 64,
                 max_side: int = 1024) -> list[dict]:
    """Batched scan: cameras with side ~ U{min..max}, a ~ U[0, 0.998],
    inclination ~ U[5, 85] deg, profiles cycled over all eight, rho0 log-uniform
    in [1e8, 1e12], 16 powerlaw_cutoff bins (1e5-1e12), inner_ring source."""
    rng = np.random.default_rng(seed)
    cams = []
    for k in range(n_cams):
        side = int(rng.integers(min_side, max_side + 1))
        cams.append(dict(nx=side, ny=side, a_spin=float(rng.uniform(0.0, 0.998)),
                         theta_obs_deg=float(rng.uniform(5.0, 85.0)),
                         profile=k % 8, rho0_gcm3=float(10.0 ** rng.uniform(8.0, 12.0)),
                         r_obs_rg=60.0, r_max_rg=120.0, fov_deg=25.0, h=0.01, max_steps=200000,
                         M_bh_msun=3.0, rho_floor_gcm3=1.0e-3, source="inner_ring",
                         spectral="powerlaw_cutoff", spec_gamma=2.0, spec_ecut_GeV=1.0e12,
                         spec_e_min_GeV=1.0e5, spec_e_max_GeV=1.0e12, n_bins=16,
                         precision="mixed", **_SOURCE_DEFAULTS))
    return cams


def production_point(**over) -> dict:
    """One parameter point of the production scan: 4096x4096 x 64 bins
    (powerlaw_cutoff 1e5-1e12), collapsar_ndaf_like (r0 12, sigma_r 8, H 0.45,
    r_min 3, r_max 80), density_weighted source, a=0.95."""
    d = dict(nx=4096, ny=4096, a_spin=0.95, theta_obs_deg=45.0, r_obs_rg=60.0, r_max_rg=120.0,
             fov_deg=25.0, h=0.01, max_steps=200000, M_bh_msun=3.0,
             profile="collapsar_ndaf_like", rho0_gcm3=1.0e11, r0_rg=12.0, sigma_r_rg=8.0,
             H_over_R=0.45, torus_r_min_rg=3.0, torus_r_max_rg=80.0, rho_floor_gcm3=1.0e-3,
             source="density_weighted", src_rho_ref_gcm3=-1.0, spectral="powerlaw_cutoff",
             spec_gamma=2.0, spec_ecut_GeV=1.0e12, spec_e_min_GeV=1.0e5, spec_e_max_GeV=1.0e12,
             n_bins=64, precision="mixed", **_SOURCE_DEFAULTS)
    d.update(over)
    return d


def strided_pixels(nx: int, ny: int, k: int) -> np.ndarray:
    """Every k-th pixel in i and j (ids j*nx+i), the CPU-baseline subset."""
    ii = np.arange(0, nx, k)
    jj = np.arange(0, ny, k)
    return (jj[:, None] * nx + ii[None, :]).ravel().astype(np.int32)


def surrogate_training_cams(n_cams: int = 128, seed: int = SEED, side: int = 2048,
                            n_bins: int = 32) -> list[dict]:
    """Surrogate training cameras in the style of mixed_512 (funnel_wall source,
    powerlaw_cutoff 1e5-1e12 GeV, mixed precision) on a side x side pixel grid,
    with a ~ U[0, 0.998], cos(inclination) ~ U[cos 85, cos 5], profile ~ U over
    all eight, rho0 log-uniform in [1e8, 1e12] (envelope 0.01 rho0), and the two
    shape parameters r0 ~ U[6, 14] M and H/R ~ U[0.15, 0.45]."""
    rng = np.random.default_rng(seed)
    lo, hi = math.cos(math.radians(85.0)), math.cos(math.radians(5.0))
    cams = []
    for _ in range(n_cams):
        rho0 = float(10.0 ** rng.uniform(8.0, 12.0))
        cams.append(mixed_512(nx=side, ny=side, n_bins=n_bins, a_spin=float(rng.uniform(0.0, 0.998)),
                              theta_obs_deg=math.degrees(math.acos(rng.uniform(lo, hi))),
                              profile=int(rng.integers(0, 8)), rho0_gcm3=rho0, envelope_rho0_gcm3=0.01 * rho0,
                              r0_rg=float(rng.uniform(6.0, 14.0)), H_over_R=float(rng.uniform(0.15, 0.45))))
    return cams


def surrogate_inference_image(**over) -> dict:
    """The surrogate's inference image: mixed_512's camera and medium at
    2048 x 2048 pixels and 32 bins."""
    d = mixed_512(nx=2048, ny=2048, n_bins=32)
    d.update(over)
    return d


def scan_points(n: int = 256, seed: int = SEED) -> list[tuple[float, float]]:
    """Production-scan parameter points: (rho0 log-uniform in [1e9, 1e12],
    inclination ~ U[10, 80] deg)."""
    rng = np.random.default_rng(seed)
    return [(float(10.0 ** rng.uniform(9.0, 12.0)), float(rng.uniform(10.0, 80.0))) for _ in range(n)]
