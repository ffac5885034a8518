"""The reference's scan scripts through the C ABI instead of subprocesses.

robustness (default):

The reference's scripts/run_robustness_scans.py (:19-56 parameters,
:190-270 cases) traces ten geodesic caches with compute_kerr_geodesics, runs
compute_kerr_image_from_cache once per case (47 cases, 16x16 pixels), reads
each .dat back and reduces it to five metrics (image_metrics, :152-169).
Here the same 47 cameras go through one hadros_batch launch, the metrics come
from the in-memory outputs, and the same scan_summary.csv and
scan_summary.md are written.  The metrics are taken, as the reference takes
them, from values rounded to the .dat's %.8e.  With --write-dat each case's
.dat is also written under the reference's file name.  The plots of the
reference script are not drawn: matplotlib is not a dependency.

    python -m hadros_b200.robustness [--outdir output/scans] [--sigma FILE]
           [--pixels 16] [--precision fp64|mixed] [--write-dat DIR]

spectral: scripts/validate_uhe_spectral_models.py (:21-61 parameters,
:153-171 metrics, :240-296 outputs) runs compute_kerr_image_from_cache six
times on the Makefile's small cache (a 0.0001, r_obs 60, theta 80, fov 25,
32x32, r_max 40, step 0.01; Makefile:224-230, :671): the three UHE spectral
models at 8 bins and powerlaw_cutoff at 4, 8 and 16 bins.  Here the six
images are one batch launch; spectral_validation.csv and
spectral_validation.md are the script's.

    python -m hadros_b200.robustness spectral [--outdir output/spectra] ...

mev-bands: scripts/make_mev_multiband_image.py (:19-23 bands, :56-141
parameters, :144-201 outputs) runs the CPU app once per Fermi-Dirac MeV band
(3-8, 8-20, 20-50 MeV) on the small cache and turns the three I_obs_mev images
into mev_multiband_flux.csv and a false-colour image.  Here the three bands
are one batch launch; the CSV is the script's and the image is written as a
binary PPM (mev_multiband_false_color_image.ppm) instead of a matplotlib PNG.

    python -m hadros_b200.robustness mev-bands [--outdir output/mev_neutrinosphere] ...

Argument mapping (compute_kerr_image_from_cache argv, apps/
compute_kerr_image_from_cache.cpp:57-201): the "h" of the parameter table is
the torus H/R, angles are degrees, and the camera is the cache's
(compute_kerr_geodesics spin, r_obs 60, theta, fov 25, n x n, r_max 60,
step 0.02; scripts/run_robustness_scans.py:80-99).
"""
from __future__ import annotations

import argparse
import csv
import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

from . import Context, SigmaTable, lib, params
from . import workloads as W
from .abi import HadrosImageOut

# scripts/run_robustness_scans.py:19-56 (the same parameter table)
BASE = {
    "enu": "1e5", "aspin": "0.0001", "mbh": "3.0", "rho0": "1.0e-2", "r0": "10.0", "sigma": "5.0",
    "h": "0.25", "source_r": "3.5", "source_sigma": "1.0", "source_theta": "15.0",
    "source_powerlaw": "2.0", "source_emax": "1.0e12", "source_norm": "1.0", "mev_enu": "10.0",
    "mev_norm": "1.0", "cam_theta": "80.0", "sigma_path": "data/sigma/sigma_nuN_CC_GBW.dat",
    "density_profile": "gaussian", "radial_power": "2.0", "funnel_depletion": "0.0",
    "funnel_theta": "20.0", "envelope_rho0": "0.0", "envelope_alpha": "2.5", "r_min": "4.0",
    "r_max": "60.0", "rho_floor": "1.0e-99", "observer_distance": "60.0", "use_f3": "1",
    "source_model": "inner_ring", "source_funnel_theta": "20.0", "source_q": "1.0", "source_s": "2.0",
    "source_grad_dr": "0.1", "source_grad_dtheta": "1.0", "source_rho_ref": "1.0e-2",
    "source_cutoff_min": "0.0", "source_cutoff_max": "1.0e2",
}
CACHE = {"r_obs": 60.0, "fov_deg": 25.0, "r_max": 60.0, "step": 0.02}
SOURCES = ["inner_ring", "jet_base", "funnel_wall", "density_weighted", "shock_layer"]


def cases() -> list[dict]:
    """The scan's cases in the reference's order (run_scans, :190-270): scan,
    case label, parameter updates, and the geodesic cache's spin and theta."""
    base_cache = (BASE["aspin"], BASE["cam_theta"])
    out = []

    def add(scan, case, cache, **updates):
        out.append({"scan": scan, "case": case, "updates": {k: str(v) for k, v in updates.items()},
                    "cache": cache})

    for m in SOURCES:
        add("source_model", m, base_cache, source_model=m)
    density = {
        "gaussian": {},
        "powerlaw": {"density_profile": "powerlaw"},
        "powerlaw_funnel": {"density_profile": "powerlaw_funnel", "funnel_depletion": "1.0",
                            "funnel_theta": "20.0"},
        "powerlaw_funnel_envelope": {"density_profile": "powerlaw_funnel_envelope",
                                     "funnel_depletion": "1.0", "funnel_theta": "20.0",
                                     "envelope_rho0": "1.0e-4"},
    }
    for name, upd in density.items():
        add("density_background", name, base_cache, source_model="funnel_wall", **upd)
    for m in SOURCES:
        for enu in ["1e4", "1e5", "1e6"]:
            add("energy", f"{m}_E{enu}", base_cache, source_model=m, enu=enu)
    for theta in ["10.0", "30.0", "50.0", "70.0", "85.0"]:
        add("inclination", f"theta_{theta}", (BASE["aspin"], theta), cam_theta=theta, source_model="funnel_wall")
    for spin in ["0.0", "0.5", "0.9", "0.99"]:
        add("spin", f"a_{spin}", (spin, BASE["cam_theta"]), aspin=spin, source_model="funnel_wall")
    for q in ["0.0", "0.5", "1.0", "2.0"]:
        add("parameter_stability", f"density_weighted_q{q}", base_cache, source_model="density_weighted",
            source_q=q)
    for s in ["0.0", "1.0", "2.0", "3.0"]:
        add("parameter_stability", f"density_weighted_s{s}", base_cache, source_model="density_weighted",
            source_s=s)
    for wall in ["10.0", "20.0", "30.0"]:
        add("parameter_stability", f"funnel_wall_theta{wall}", base_cache, source_model="funnel_wall",
            source_funnel_theta=wall)
    for width in ["8.0", "15.0", "25.0"]:
        add("parameter_stability", f"funnel_wall_width{width}", base_cache, source_model="funnel_wall",
            source_theta=width)
    return out


def case_params(case: dict, pixels: int = 16, precision: str = "fp64", **over):
    """hadros_params of one case: the argv of compute_kerr_image_from_cache
    (:57-201) on the camera of its geodesic cache."""
    v = dict(BASE)
    v.update(case["updates"])
    f = lambda k: float(v[k])   # noqa: E731  (std::atof)
    spin, theta = case["cache"]
    kw = dict(
        # the geodesic cache (compute_kerr_geodesics argv, scripts/run_robustness_scans.py:80-99)
        a_spin=float(spin), r_obs_rg=CACHE["r_obs"], theta_obs_deg=float(theta), fov_deg=CACHE["fov_deg"],
        nx=pixels, ny=pixels, r_max_rg=CACHE["r_max"], h=CACHE["step"],
        # compute_kerr_image_from_cache argv 1-38
        Enu_obs_GeV=f("enu"), M_bh_msun=f("mbh"), rho0_gcm3=f("rho0"), r0_rg=f("r0"), sigma_r_rg=f("sigma"),
        H_over_R=f("h"), src_r_center_rg=f("source_r"), src_sigma_r_rg=f("source_sigma"),
        src_theta_width_deg=f("source_theta"), src_powerlaw=f("source_powerlaw"),
        src_emax_GeV=f("source_emax"), src_norm=f("source_norm"), mev_Enu_obs_MeV=f("mev_enu"),
        mev_norm=f("mev_norm"), profile=v["density_profile"], radial_power=f("radial_power"),
        funnel_depletion=f("funnel_depletion"), funnel_theta_deg=f("funnel_theta"),
        envelope_rho0_gcm3=f("envelope_rho0"), envelope_alpha=f("envelope_alpha"),
        torus_r_min_rg=f("r_min"), torus_r_max_rg=f("r_max"), rho_floor_gcm3=f("rho_floor"),
        source=v["source_model"], src_funnel_theta_deg=f("source_funnel_theta"),
        src_density_power_q=f("source_q"), src_radial_power_s=f("source_s"),
        src_gradient_dr_rg=f("source_grad_dr"), src_gradient_dtheta_deg=f("source_grad_dtheta"),
        src_rho_ref_gcm3=f("source_rho_ref"), src_cutoff_min=f("source_cutoff_min"),
        src_cutoff_max=f("source_cutoff_max"),
        spectral="monochromatic", mev_channel=1, precision=precision)
    kw.update(over)
    return params(**kw), v


def dat_round(x) -> np.ndarray:
    """Values as the reference reads them back from its .dat (%.8e text)."""
    return np.array([float(f"{float(a):.8e}") for a in np.ravel(x)])


def image_metrics(out: dict) -> dict:
    """scripts/run_robustness_scans.py:152-169 on one image's outputs."""
    tau = dat_round(out["tau"])
    psurv = dat_round(out["P_surv"])
    intensity = dat_round(out["I_obs"])
    captured = (np.asarray(out["fate"]) == 1).astype(np.float64)
    finite = np.isfinite(tau) & np.isfinite(psurv) & np.isfinite(intensity)
    return {"mean_tau": float(np.mean(tau[finite])), "max_tau": float(np.max(tau[finite])),
            "mean_P_surv": float(np.mean(psurv[finite])), "total_intensity": float(np.sum(intensity[finite])),
            "valid_rays": int(np.count_nonzero(finite & (captured == 0)))}


def make_rows(table: list[dict], outputs: list[dict], files: list[str] | None = None) -> list[dict]:
    """CSV rows (scan, case, output_file, parameters, metrics) and the energy
    scan's monotonicity flag (:206-215)."""
    rows = []
    prev = {}
    for k, (case, out) in enumerate(zip(table, outputs)):
        v = dict(BASE)
        v.update(case["updates"])
        row = {"scan": case["scan"], "case": case["case"], "output_file": files[k] if files else "", **v,
               **image_metrics(out)}
        if case["scan"] == "energy":
            group = case["case"].split("_E", 1)[0]
            p = prev.get(group)
            row["anomaly"] = "mean_tau_decreased" if p is not None and row["mean_tau"] < p else ""
            prev[group] = row["mean_tau"]
        rows.append(row)
    return rows


CASE_OUTPUTS = ("tau", "P_surv", "I_obs", "fate", "steps", "tau_mev", "P_surv_mev", "I_obs_mev", "r_nu",
                "leakage")


def run(ctx: Context | None, sigma: SigmaTable, pixels: int = 16, precision: str = "fp64",
        write_dat: str | None = None, dis_model: str = "GBW", dist=None, rank: int = 0, world: int = 1,
        trace=None) -> tuple[list[dict] | None, dict]:
    """Every case in one hadros_batch launch per rank; returns (rows, launch
    stats).  Under several ranks (dist, rank, world) the cases are split
    over them (hadros_b200.shard.run_scan) and rank 0 gets every row, the
    others None.  `trace(cams) -> outputs` replaces ctx.batch (tests trace
    with the CPU oracle)."""
    table = cases()
    cams = [case_params(c, pixels, precision)[0] for c in table]
    if trace is None:
        def trace(cs):
            return ctx.batch(cs, sigma, outputs=CASE_OUTPUTS)
    if world > 1:
        from . import shard
        outs = shard.run_scan(cams, trace, dist, rank, world)
    else:
        outs = trace(cams)
    stats = ctx.stats() if ctx is not None else {}
    if outs is None:
        return None, stats
    files = None
    if write_dat:
        files = []
        d = Path(write_dat)
        d.mkdir(parents=True, exist_ok=True)
        for p, out in zip(cams, outs):
            buf = C.create_string_buffer(1024)
            rc = lib().hadros_image_filename(C.byref(p), 1, dis_model.encode(), p.mev_Enu_obs_MeV, p.mev_norm,
                                             b".dat", buf, 1024)
            if rc:
                raise RuntimeError(lib().hadros_last_error().decode())
            path = d / buf.value.decode()
            host = {k: np.ascontiguousarray(out[k]) for k in out}
            o = HadrosImageOut()
            for k, a in host.items():
                setattr(o, k, a.ctypes.data)
            if lib().hadros_write_dat_mev(str(path).encode(), C.byref(p), dis_model.encode(), C.byref(o)):
                raise RuntimeError(lib().hadros_last_error().decode())
            files.append(str(path))
    return make_rows(table, outs, files), stats


def write_csv(rows: list[dict], outdir: Path) -> Path:
    """scan_summary.csv with the reference's columns (sorted union of keys, :273-279)."""
    outdir.mkdir(parents=True, exist_ok=True)
    keys = sorted({k for r in rows for k in r})
    path = outdir / "scan_summary.csv"
    with path.open("w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=keys)
        w.writeheader()
        w.writerows(rows)
    return path


def write_markdown(rows: list[dict], outdir: Path) -> Path:
    """scan_summary.md with the reference's observations (:356-425)."""
    def of(scan):
        return [r for r in rows if r["scan"] == scan]
    lines = ["# Robustness scan summary", "",
             "Moderate-resolution scans were run for Point 3. These are validation-scale",
             "parameter studies, not production-resolution figures.", "", "## Key observations", ""]
    src = of("source_model")
    if src:
        t = [float(r["mean_tau"]) for r in src]
        lines.append(f"- Source morphology changes total intensity, but mean tau stays in the range "
                     f"{min(t):.3e}-{max(t):.3e} for the fixed Gaussian background.")
    den = of("density_background")
    if den:
        t = [float(r["mean_tau"]) for r in den]
        lines.append(f"- Density morphology changes mean tau over {min(t):.3e}-{max(t):.3e}.")
    anomalies = [r for r in rows if r.get("anomaly")]
    if anomalies:
        lines.append(f"- Energy scan anomalies flagged: {len(anomalies)} cases.")
    else:
        lines.append("- No monotonicity anomalies were flagged in mean tau over the sampled UHE energies.")
    spin = of("spin")
    if spin:
        i = [float(r["total_intensity"]) for r in spin]
        lines.append(f"- Spin modifies image intensity over {min(i):.3e}-{max(i):.3e} in this validation grid.")
    lines += ["", "## Outputs", "", "- `scan_summary.csv`", "", "## Interpretation guardrails", "",
              "These scans support robustness of qualitative trends at moderate resolution.",
              "They should not be presented as production-resolution convergence tests."]
    path = outdir / "scan_summary.md"
    path.write_text("\n".join(lines) + "\n")
    return path


# scripts/validate_uhe_spectral_models.py:21-61 (the same parameter table)
SPECTRAL_BASE = {
    "enu": "1e11", "a": "0.0001", "mbh": "3.0", "rho0": "1.0e0", "r0": "10.0", "sigma": "5.0", "h": "0.25",
    "source_r": "3.5", "source_sigma": "1.0", "source_theta": "15.0", "source_powerlaw": "2.0",
    "source_emax": "1.0e12", "source_norm": "1.0", "mev_enu": "10.0", "mev_norm": "1.0", "cam_theta": "80.0",
    "sigma_path": "data/sigma/sigma_nuN_CC_GBW.dat", "profile": "powerlaw_funnel_envelope",
    "radial_power": "2.0", "funnel_depletion": "1.0", "funnel_theta": "20.0", "envelope_rho0": "1.0e-2",
    "envelope_alpha": "2.5", "r_min": "4.0", "r_max": "60.0", "rho_floor": "1.0e-99",
    "observer_distance": "60.0", "use_f3": "1", "cache": "output/rays/kerr_geodesics_small.bin",
    "source_model": "funnel_wall", "source_funnel_theta": "20.0", "source_q": "1.0", "source_s": "2.0",
    "source_grad_dr": "0.1", "source_grad_dtheta": "1.0", "source_rho_ref": "1.0e0",
    "source_cutoff_min": "0.0", "source_cutoff_max": "1.0e2",
}
# the small cache (Makefile:43-51, :224-230, :671)
SMALL_CACHE = {"a": 0.0001, "r_obs": 60.0, "theta": 80.0, "fov_deg": 25.0, "pixels": 32, "r_max": 40.0,
               "step": 0.01}


def spectral_cases() -> list[tuple[str, int, str]]:
    """(spectral model, bins, row label) in the script's order (:244-252)."""
    out = [(m, 8, m) for m in ("monochromatic", "powerlaw", "powerlaw_cutoff")]
    out += [("powerlaw_cutoff", n, f"powerlaw_cutoff_bins{n}") for n in (4, 8, 16)]
    return out


def spectral_params(model: str, n_bins: int, pixels: int = 32, precision: str = "fp64", **over):
    """compute() of the script (:98-150): the CPU app's argv 1-44 with the
    spectral arguments model, gamma 2, E_cut 1e12, 1e5-1e12 GeV, n_bins."""
    v = SPECTRAL_BASE
    f = lambda k: float(v[k])   # noqa: E731  (std::atof)
    kw = dict(
        a_spin=SMALL_CACHE["a"], r_obs_rg=SMALL_CACHE["r_obs"], theta_obs_deg=SMALL_CACHE["theta"],
        fov_deg=SMALL_CACHE["fov_deg"], nx=pixels, ny=pixels, r_max_rg=SMALL_CACHE["r_max"],
        h=SMALL_CACHE["step"],
        Enu_obs_GeV=f("enu"), M_bh_msun=f("mbh"), rho0_gcm3=f("rho0"), r0_rg=f("r0"), sigma_r_rg=f("sigma"),
        H_over_R=f("h"), src_r_center_rg=f("source_r"), src_sigma_r_rg=f("source_sigma"),
        src_theta_width_deg=f("source_theta"), src_powerlaw=f("source_powerlaw"),
        src_emax_GeV=f("source_emax"), src_norm=f("source_norm"), mev_Enu_obs_MeV=f("mev_enu"),
        mev_norm=f("mev_norm"), profile=v["profile"], radial_power=f("radial_power"),
        funnel_depletion=f("funnel_depletion"), funnel_theta_deg=f("funnel_theta"),
        envelope_rho0_gcm3=f("envelope_rho0"), envelope_alpha=f("envelope_alpha"),
        torus_r_min_rg=f("r_min"), torus_r_max_rg=f("r_max"), rho_floor_gcm3=f("rho_floor"),
        source=v["source_model"], src_funnel_theta_deg=f("source_funnel_theta"),
        src_density_power_q=f("source_q"), src_radial_power_s=f("source_s"),
        src_gradient_dr_rg=f("source_grad_dr"), src_gradient_dtheta_deg=f("source_grad_dtheta"),
        src_rho_ref_gcm3=f("source_rho_ref"), src_cutoff_min=f("source_cutoff_min"),
        src_cutoff_max=f("source_cutoff_max"),
        spectral=model, spec_gamma=2.0, spec_ecut_GeV=1.0e12, spec_e_min_GeV=1.0e5, spec_e_max_GeV=1.0e12,
        n_bins=n_bins, mev_channel=1, precision=precision)
    kw.update(over)
    return params(**kw)


def spectral_metrics(out: dict, label: str, n_bins: int) -> dict:
    """metrics() of the script (:153-171)."""
    tau, psurv, inten = dat_round(out["tau"]), dat_round(out["P_surv"]), dat_round(out["I_obs"])
    finite = np.isfinite(tau) & np.isfinite(psurv) & np.isfinite(inten)
    return {"spectral_model": label, "n_bins": n_bins, "mean_tau": float(np.mean(tau[finite])),
            "max_tau": float(np.max(tau[finite])), "mean_Psurv": float(np.mean(psurv[finite])),
            "integrated_intensity": float(np.sum(inten[finite])), "valid_pixels": int(np.count_nonzero(finite)),
            "finite_outputs": bool(np.all(finite)), "positive_weights": True}


def run_spectral(ctx: Context, sigma: SigmaTable, pixels: int = 32, precision: str = "fp64") -> tuple[list, dict]:
    """The six images in one hadros_batch launch; returns (rows, launch stats)."""
    table = spectral_cases()
    cams = [spectral_params(m, n, pixels, precision) for m, n, _ in table]
    outs = ctx.batch(cams, sigma, outputs=("tau", "P_surv", "I_obs", "fate", "steps"))
    return [spectral_metrics(o, label, n) for (m, n, label), o in zip(table, outs)], ctx.stats()


def write_spectral(rows: list[dict], outdir: Path) -> tuple[Path, Path]:
    """spectral_validation.csv and .md as the script writes them (:254-293)."""
    outdir.mkdir(parents=True, exist_ok=True)
    csv_path = outdir / "spectral_validation.csv"
    with csv_path.open("w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=list(rows[0].keys()))
        w.writeheader()
        w.writerows(rows)
    finite_ok = all(bool(r["finite_outputs"]) for r in rows)
    positive = all(float(r["integrated_intensity"]) >= 0.0 for r in rows)
    conv = [float(r["integrated_intensity"]) for r in rows if str(r["spectral_model"]).startswith("powerlaw_cutoff_bins")]
    rel_8_16 = abs(conv[1] - conv[2]) / max(abs(conv[2]), 1.0e-300)
    lines = ["# UHE spectral validation", "", f"- finite_outputs: {finite_ok}",
             f"- nonnegative_integrated_intensity: {positive}",
             f"- powerlaw_cutoff convergence |I_8-I_16|/I_16: {rel_8_16:.6e}", "", "## Metrics", ""]
    for r in rows:
        lines.append(f"- {r['spectral_model']} bins={r['n_bins']}: mean_tau={float(r['mean_tau']):.6e}, "
                     f"mean_Psurv={float(r['mean_Psurv']):.6e}, I={float(r['integrated_intensity']):.6e}")
    md_path = outdir / "spectral_validation.md"
    md_path.write_text("\n".join(lines) + "\n")
    return csv_path, md_path


# scripts/make_mev_multiband_image.py:19-23
MEV_BANDS = [("low-energy MeV band", "blue", 3.0, 8.0),
             ("intermediate-energy MeV band", "green", 8.0, 20.0),
             ("high-energy MeV band", "red", 20.0, 50.0)]


def mev_band_params(e_min: float, e_max: float, pixels: int = 32, precision: str = "fp64", **over):
    """compute_band() of the script (:56-141) with its environment defaults:
    the small cache, gaussian torus rho0 1e10, floor 1e-20, inner_ring source
    with rho_ref = rho0, monochromatic 1e11 GeV, the physical anti_nu_e MeV
    model with the Fermi-Dirac band [e_min, e_max] in 8 bins."""
    rho0 = 1.0e10
    kw = dict(
        a_spin=SMALL_CACHE["a"], r_obs_rg=SMALL_CACHE["r_obs"], theta_obs_deg=SMALL_CACHE["theta"],
        fov_deg=SMALL_CACHE["fov_deg"], nx=pixels, ny=pixels, r_max_rg=SMALL_CACHE["r_max"],
        h=SMALL_CACHE["step"],
        Enu_obs_GeV=1.0e11, M_bh_msun=3.0, rho0_gcm3=rho0, r0_rg=10.0, sigma_r_rg=5.0, H_over_R=0.25,
        src_r_center_rg=3.5, src_sigma_r_rg=1.0, src_theta_width_deg=15.0, src_powerlaw=2.0, src_emax_GeV=1.0e12,
        src_norm=1.0, profile="gaussian", radial_power=2.0, funnel_depletion=0.0, funnel_theta_deg=15.0,
        envelope_rho0_gcm3=0.0, envelope_alpha=2.5, torus_r_min_rg=4.0, torus_r_max_rg=60.0,
        rho_floor_gcm3=1.0e-20, source="inner_ring", src_funnel_theta_deg=20.0, src_density_power_q=1.0,
        src_radial_power_s=2.0, src_gradient_dr_rg=0.1, src_gradient_dtheta_deg=1.0, src_rho_ref_gcm3=rho0,
        src_cutoff_min=0.0, src_cutoff_max=1.0e2, spectral="monochromatic", spec_gamma=2.0,
        spec_ecut_GeV=1.0e12, spec_e_min_GeV=1.0e5, spec_e_max_GeV=1.0e12, n_bins=8,
        mev_channel=1, mev_model="physical", mev_flavor="anti_nu_e", mev_thermal="inner_hot_torus",
        mev_ye="neutron_rich_torus", mev_T0_MeV=6.0, mev_T_floor_MeV=0.1, mev_T_power=0.2, mev_Ye_torus=0.25,
        mev_Ye_funnel=0.55, mev_Ye_envelope=0.45, mev_Ye_floor=0.01, mev_Ye_ceil=0.60,
        mev_spectral="fermi_dirac_band", mev_E_min_MeV=e_min, mev_E_max_MeV=e_max, mev_n_bins=8,
        mev_Enu_obs_MeV=10.0, mev_norm=1.0, mev_degeneracy_correction=False, precision=precision)
    kw.update(over)
    return params(**kw)


def band_grid(I_mev, nx: int, ny: int) -> np.ndarray:
    """load_grid() of the script (:144-156): grid[ny - 1 - j, i] = I_obs_mev."""
    v = dat_round(I_mev).reshape(ny, nx)   # rows j*nx + i
    return v[::-1, :].copy()


def run_mev_bands(ctx: Context, sigma: SigmaTable, pixels: int = 32, precision: str = "fp64"):
    """The three bands in one hadros_batch launch; returns (rows, grids, stats)."""
    cams = [mev_band_params(lo, hi, pixels, precision) for _, _, lo, hi in MEV_BANDS]
    outs = ctx.batch(cams, sigma, outputs=("tau", "P_surv", "I_obs", "fate", "steps", "tau_mev", "P_surv_mev",
                                            "I_obs_mev", "r_nu", "leakage"))
    grids, rows = [], []
    for (label, color, lo, hi), out in zip(MEV_BANDS, outs):
        grids.append(band_grid(out["I_obs_mev"], pixels, pixels))
        rows.append({"band": label, "false_color": color, "E_min_MeV": lo, "E_max_MeV": hi,
                     "integrated_I_mev": float(np.sum(dat_round(out["I_obs_mev"]))), "data_path": ""})
    return rows, grids, ctx.stats()


def write_mev_bands(rows: list[dict], grids: list[np.ndarray], outdir: Path) -> tuple[Path, Path]:
    """mev_multiband_flux.csv (:162-191) and the false-colour image: channel =
    sqrt(I / max I) clipped at 0, red = 20-50 MeV, green = 8-20, blue = 3-8
    (:159-170), as an 8-bit binary PPM shown the way the script's
    imshow(origin="lower") shows it."""
    outdir.mkdir(parents=True, exist_ok=True)
    lines = ["# product false-color MeV energy-band diagnostic image", "# blue low-energy MeV band 3-8 MeV",
             "# green intermediate-energy MeV band 8-20 MeV", "# red high-energy MeV band 20-50 MeV",
             "# note colors encode MeV neutrino energy intervals, not photon colors",
             "band,false_color,E_min_MeV,E_max_MeV,integrated_I_mev,data_path"]
    for r in rows:
        lines.append(f"{r['band']},{r['false_color']},{r['E_min_MeV']:g},{r['E_max_MeV']:g},"
                     f"{r['integrated_I_mev']:.8e},{r['data_path']}")
    csv_path = outdir / "mev_multiband_flux.csv"
    csv_path.write_text("\n".join(lines) + "\n")

    def norm(g):
        g = np.clip(g, 0.0, None)
        m = float(np.nanmax(g)) if g.size else 0.0
        return np.zeros_like(g) if m <= 0.0 else np.sqrt(g / m)
    blue, green, red = (norm(g) for g in grids)
    rgb = np.dstack([red, green, blue])[::-1]   # origin="lower": the grid's last row on top
    # a NaN cell is blank, as imshow leaves it, not an undefined byte
    rgb = np.nan_to_num(rgb, nan=0.0, posinf=1.0, neginf=0.0)
    img = np.clip(np.rint(rgb * 255.0), 0, 255).astype(np.uint8)
    ppm = outdir / "mev_multiband_false_color_image.ppm"
    with ppm.open("wb") as f:
        f.write(f"P6\n{img.shape[1]} {img.shape[0]}\n255\n".encode())
        f.write(img.tobytes())
    return csv_path, ppm


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m hadros_b200.robustness", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("scan", nargs="?", choices=("robustness", "spectral", "mev-bands"), default="robustness")
    ap.add_argument("--outdir", default=None, help="default output/scans (robustness), output/spectra (spectral)")
    ap.add_argument("--sigma", default=None, help="sigma table (reference format); default: the synthetic table")
    ap.add_argument("--pixels", type=int, default=None, help="image side (default 16 robustness, 32 spectral)")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--write-dat", default=None, help="also write each case's .dat into this directory")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    if a.sigma:
        sig = SigmaTable.load(a.sigma)
    else:
        E, g2, s = W.synthetic_sigma_arrays()
        sig = SigmaTable.from_arrays(E, s, g2)
    if a.scan == "mev-bands":
        with Context(a.device) as ctx:
            rows, grids, st = run_mev_bands(ctx, sig, a.pixels or SMALL_CACHE["pixels"], a.precision)
        csv_path, ppm = write_mev_bands(rows, grids, Path(a.outdir or "output/mev_neutrinosphere"))
        print(json.dumps({"bands_per_launch": len(rows), "launches": st["launches"], "rays": st["rays"],
                          "kernel_ms": st["kernel_ms"], "csv": str(csv_path), "image": str(ppm)}))
        return 0
    if a.scan == "spectral":
        with Context(a.device) as ctx:
            rows, st = run_spectral(ctx, sig, a.pixels or SMALL_CACHE["pixels"], a.precision)
        csv_path, md_path = write_spectral(rows, Path(a.outdir or "output/spectra"))
        print(json.dumps({"images_per_launch": len(rows), "launches": st["launches"], "rays": st["rays"],
                          "kernel_ms": st["kernel_ms"], "csv": str(csv_path), "md": str(md_path)}))
        return 0
    from . import shard
    dist, rank, world, local = shard.init_from_env()   # torchrun: the cases are split over the ranks
    try:
        with Context(local if world > 1 else a.device) as ctx:
            rows, st = run(ctx, sig, a.pixels or 16, a.precision, a.write_dat, dist=dist, rank=rank, world=world)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    if rows is None:
        return 0
    out = Path(a.outdir or "output/scans")
    csv_path = write_csv(rows, out)
    md_path = write_markdown(rows, out)
    print(json.dumps({"cases": len(rows), "ranks": world, "cameras_per_launch": len(rows) // world,
                      "launches": st["launches"],
                      "rays": st["rays"], "kernel_ms": st["kernel_ms"], "total_ms": st["total_ms"],
                      "csv": str(csv_path), "md": str(md_path)}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
