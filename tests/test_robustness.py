"""hadros_b200.robustness: the reference's robustness scan
(scripts/run_robustness_scans.py) and spectral validation
(scripts/validate_uhe_spectral_models.py) through the C ABI.  CPU tests: the
case tables, the argv mapping, and our rows against the reference's own two
executables run the way the scripts run them (where oracle/build_ref.sh built
them).  The GPU runs are in test_gpu_robustness.py."""
from __future__ import annotations

import collections
import math
import subprocess

import numpy as np
import pytest

from conftest import ROOT

REF_DIR = ROOT / "oracle" / "_ref"
REF_GEO = REF_DIR / "compute_kerr_geodesics"
REF_IMG = REF_DIR / "compute_kerr_image_from_cache"


def test_case_table_is_the_reference_scan():
    from hadros_b200 import robustness as R
    t = R.cases()
    assert len(t) == 47
    assert collections.Counter(c["scan"] for c in t) == {
        "source_model": 5, "density_background": 4, "energy": 15, "inclination": 5, "spin": 4,
        "parameter_stability": 14}
    assert [c["case"] for c in t[:5]] == ["inner_ring", "jet_base", "funnel_wall", "density_weighted",
                                          "shock_layer"]
    assert t[9]["case"] == "inner_ring_E1e4" and t[9]["updates"] == {"source_model": "inner_ring", "enu": "1e4"}
    caches = {c["cache"] for c in t}
    assert len(caches) == 10   # the ten geodesic caches the script makes


def test_case_params_follow_the_cpu_app_argv(hb):
    from hadros_b200 import robustness as R
    t = {(c["scan"], c["case"]): c for c in R.cases()}
    p, v = R.case_params(t[("density_background", "powerlaw_funnel_envelope")])
    assert (p.nx, p.ny, p.h, p.r_max_rg, p.r_obs_rg, p.fov_deg) == (16, 16, 0.02, 60.0, 60.0, 25.0)
    assert p.H_over_R == 0.25 and p.sigma_r_rg == 5.0 and p.r0_rg == 10.0 and p.rho0_gcm3 == 1.0e-2
    assert p.profile_kind == hb.PROFILES.index("powerlaw_funnel_envelope")
    assert p.source_kind == hb.SOURCES.index("funnel_wall")
    assert p.funnel_depletion == 1.0 and p.envelope_rho0_gcm3 == 1.0e-4
    assert p.theta_obs_rad == 80.0 * math.pi / 180.0 and p.src_theta_width_rad == 15.0 * math.pi / 180.0
    assert p.a_spin == 0.0001 and p.Enu_obs_GeV == 1.0e5 and p.mev_channel == 1
    q, _ = R.case_params(t[("spin", "a_0.99")])
    assert q.a_spin == 0.99
    w, _ = R.case_params(t[("parameter_stability", "funnel_wall_width25.0")])
    assert w.src_theta_width_rad == 25.0 * math.pi / 180.0


def _ref_image_args(R, case, cache, sigma_path):
    """scripts/run_robustness_scans.py:101-141 with this machine's sigma file."""
    v = dict(R.BASE)
    v.update(case["updates"])
    v["sigma_path"] = str(sigma_path)
    keys = ["enu", "aspin", "mbh", "rho0", "r0", "sigma", "h", "source_r", "source_sigma", "source_theta",
            "source_powerlaw", "source_emax", "source_norm", "mev_enu", "mev_norm", "cam_theta", "sigma_path",
            "density_profile", "radial_power", "funnel_depletion", "funnel_theta", "envelope_rho0",
            "envelope_alpha", "r_min", "r_max", "rho_floor", "observer_distance", "use_f3"]
    tail = ["source_model", "source_funnel_theta", "source_q", "source_s", "source_grad_dr", "source_grad_dtheta",
            "source_rho_ref", "source_cutoff_min", "source_cutoff_max"]
    return [str(REF_IMG)] + [v[k] for k in keys] + [str(cache)] + [v[k] for k in tail]


@pytest.mark.skipif(not (REF_GEO.exists() and REF_IMG.exists()), reason="reference executables not built here")
def test_rows_equal_the_reference_executables(hb, tmp_path, sigma_arrays):
    """Three cases at 4x4 pixels run as the script runs them
    (compute_kerr_geodesics, then compute_kerr_image_from_cache, then the
    .dat read back): our rows, built from the oracle's in-memory outputs, give
    the same five metrics, and the .dat's MeV columns are the oracle's."""
    from hadros_b200 import robustness as R
    from hadros_b200 import workloads as W
    from oracle import pyoracle as O
    E, g2, s = sigma_arrays
    sig = tmp_path / "sigma.dat"
    W.write_sigma_file(sig, E, g2, s)
    (tmp_path / "output" / "images").mkdir(parents=True)
    table = {(c["scan"], c["case"]): c for c in R.cases()}
    picks = [table[("source_model", "funnel_wall")], table[("energy", "jet_base_E1e6")],
             table[("spin", "a_0.9")]]
    for case in picks:
        spin, theta = case["cache"]
        cache = tmp_path / f"cache_{spin}_{theta}.bin"
        r = subprocess.run([str(REF_GEO), spin, "60.0", theta, "25.0", "4", "4", "60.0", "0.02", str(cache)],
                           capture_output=True, text=True, timeout=600, env={"OMP_NUM_THREADS": "4"})
        assert r.returncode == 0, r.stderr
        r = subprocess.run(_ref_image_args(R, case, cache, sig), cwd=tmp_path, capture_output=True, text=True,
                           timeout=600, env={"OMP_NUM_THREADS": "4"})
        assert r.returncode == 0, r.stderr
        saved = [ln.split("Saved: ", 1)[1] for ln in r.stdout.splitlines()
                 if ln.startswith("Saved: ") and ln.endswith(".dat")]
        data = np.loadtxt(tmp_path / saved[0], comments="#")
        tau, psurv, inten, captured = data[:, 4], data[:, 5], data[:, 6], data[:, 7]
        finite = np.isfinite(tau) & np.isfinite(psurv) & np.isfinite(inten)
        theirs = {"mean_tau": np.mean(tau[finite]), "max_tau": np.max(tau[finite]),
                  "mean_P_surv": np.mean(psurv[finite]), "total_intensity": np.sum(inten[finite]),
                  "valid_rays": int(np.count_nonzero(finite & (captured == 0)))}
        p, _ = R.case_params(case, pixels=4)
        ref = O.oracle_image(p, E, s, mev=True)
        row = R.make_rows([case], [ref])[0]
        for k in ("mean_tau", "max_tau", "mean_P_surv", "total_intensity"):
            assert row[k] == pytest.approx(theirs[k], rel=1e-12, abs=0.0), (case["case"], k)
        assert row["valid_rays"] == theirs["valid_rays"]
        for c, key in enumerate(O.MEV_KEYS):   # .dat rows are in cache order: key them by pixel
            for line in data:
                k = int(line[1]) * 4 + int(line[0])
                assert line[8 + c] == pytest.approx(ref[key][k], rel=1e-8, abs=1e-300), (case["case"], key)


def test_spectral_table_and_params(hb):
    from hadros_b200 import robustness as R
    t = R.spectral_cases()
    assert [x[2] for x in t] == ["monochromatic", "powerlaw", "powerlaw_cutoff", "powerlaw_cutoff_bins4",
                                 "powerlaw_cutoff_bins8", "powerlaw_cutoff_bins16"]
    p = R.spectral_params("powerlaw_cutoff", 16)
    assert (p.nx, p.r_max_rg, p.h, p.a_spin, p.fov_deg) == (32, 40.0, 0.01, 0.0001, 25.0)
    assert p.spectral_kind == 2 and p.n_bins == 16 and p.spec_e_min_GeV == 1.0e5 and p.spec_ecut_GeV == 1.0e12
    assert p.rho0_gcm3 == 1.0 and p.envelope_rho0_gcm3 == 1.0e-2 and p.src_rho_ref_gcm3 == 1.0


@pytest.mark.skipif(not (REF_GEO.exists() and REF_IMG.exists()), reason="reference executables not built here")
def test_spectral_rows_equal_the_reference_executables(hb, tmp_path, sigma_arrays):
    """validate_uhe_spectral_models.py's compute() + metrics() for the
    powerlaw_cutoff case on a 4x4 small cache, against our row from the
    oracle's outputs."""
    from hadros_b200 import robustness as R
    from hadros_b200 import workloads as W
    from oracle import pyoracle as O
    E, g2, s = sigma_arrays
    sig = tmp_path / "sigma.dat"
    W.write_sigma_file(sig, E, g2, s)
    (tmp_path / "output" / "images").mkdir(parents=True)
    cache = tmp_path / "small.bin"
    r = subprocess.run([str(REF_GEO), "0.0001", "60.0", "80.0", "25.0", "4", "4", "40.0", "0.01", str(cache)],
                       capture_output=True, text=True, timeout=600, env={"OMP_NUM_THREADS": "4"})
    assert r.returncode == 0, r.stderr
    v = dict(R.SPECTRAL_BASE, sigma_path=str(sig), cache=str(cache))
    keys = ["enu", "a", "mbh", "rho0", "r0", "sigma", "h", "source_r", "source_sigma", "source_theta",
            "source_powerlaw", "source_emax", "source_norm", "mev_enu", "mev_norm", "cam_theta", "sigma_path",
            "profile", "radial_power", "funnel_depletion", "funnel_theta", "envelope_rho0", "envelope_alpha",
            "r_min", "r_max", "rho_floor", "observer_distance", "use_f3", "cache", "source_model",
            "source_funnel_theta", "source_q", "source_s", "source_grad_dr", "source_grad_dtheta",
            "source_rho_ref", "source_cutoff_min", "source_cutoff_max"]
    argv = [str(REF_IMG)] + [v[k] for k in keys] + ["powerlaw_cutoff", "2.0", "1.0e12", "1.0e5", "1.0e12", "4"]
    r = subprocess.run(argv, cwd=tmp_path, capture_output=True, text=True, timeout=600,
                       env={"OMP_NUM_THREADS": "4"})
    assert r.returncode == 0, r.stderr
    saved = [ln.split("Saved: ", 1)[1] for ln in r.stdout.splitlines() if ln.startswith("Saved: ")]
    data = np.loadtxt(tmp_path / saved[0])
    tau, psurv, inten = data[:, 4], data[:, 5], data[:, 6]
    ours = R.spectral_metrics(O.oracle_image(R.spectral_params("powerlaw_cutoff", 4, pixels=4), E, s),
                              "powerlaw_cutoff_bins4", 4)
    assert ours["mean_tau"] == pytest.approx(np.mean(tau), rel=1e-12)
    assert ours["max_tau"] == pytest.approx(np.max(tau), rel=1e-12)
    assert ours["mean_Psurv"] == pytest.approx(np.mean(psurv), rel=1e-12)
    assert ours["integrated_intensity"] == pytest.approx(np.sum(inten), rel=1e-12, abs=0.0)
    assert ours["valid_pixels"] == 16 and ours["finite_outputs"]


class _OracleContext:
    """Context.batch / Context.stats answered by the CPU oracle, so the scan
    modules' host logic runs without a GPU."""

    def __init__(self, E, s):
        self.E, self.s, self.rays = E, s, 0

    def batch(self, cams, sigma, outputs):
        from oracle import pyoracle as O
        self.rays = sum(int(c.nx) * int(c.ny) for c in cams)
        return [O.oracle_image(c, self.E, self.s, mev=True) for c in cams]

    def stats(self):
        return {"launches": 1, "rays": self.rays, "kernel_ms": 0.0}


@pytest.mark.skipif(not (REF_GEO.exists() and REF_IMG.exists()), reason="reference executables not built here")
def test_mev_bands_equal_the_reference_executables(hb, tmp_path, sigma_arrays):
    """make_mev_multiband_image.py's compute_band() for the 8-20 MeV band on a
    4x4 small cache, run as the script runs it (71 arguments), against the
    module's row; the CSV and the PPM image it writes."""
    from hadros_b200 import robustness as R
    from hadros_b200 import workloads as W
    E, g2, s = sigma_arrays
    sig = tmp_path / "sigma.dat"
    W.write_sigma_file(sig, E, g2, s)
    (tmp_path / "output" / "images").mkdir(parents=True)
    cache = tmp_path / "small.bin"
    r = subprocess.run([str(REF_GEO), "0.0001", "60.0", "80.0", "25.0", "4", "4", "40.0", "0.01", str(cache)],
                       capture_output=True, text=True, timeout=600, env={"OMP_NUM_THREADS": "4"})
    assert r.returncode == 0, r.stderr
    argv = [str(REF_IMG), "100000000000.0", "0.0001", "3.0", "10000000000.0", "10.0", "5.0", "0.25", "3.5", "1.0",
            "15.0", "2.0", "1.0e12", "1.0", "10.0", "1.0", "80.0", str(sig), "gaussian", "2.0", "0.0", "15.0",
            "0.0", "2.5", "4.0", "60.0", "1.0e-20", "60.0", "1", str(cache), "inner_ring", "20.0", "1.0", "2.0",
            "0.1", "1.0", "10000000000.0", "0.0", "1.0e2", "monochromatic", "2.0", "1.0e12", "1.0e5", "1.0e12",
            "8", "physical", "anti_nu_e", "1", "1", "1", "1", "1", "inner_hot_torus", "neutron_rich_torus", "6.0",
            "0.1", "0.2", "0.25", "0.55", "0.45", "0.01", "0.60", "fermi_dirac_band", "8.0", "20.0", "8", "0", "1",
            "1", "1", "1", "1"]
    r = subprocess.run(argv, cwd=tmp_path, capture_output=True, text=True, timeout=600,
                       env={"OMP_NUM_THREADS": "4"})
    assert r.returncode == 0, r.stderr
    saved = [ln.split("Saved: ", 1)[1] for ln in r.stdout.splitlines() if ln.startswith("Saved: ")]
    assert "_MeVSpectrum_fermi_dirac_band_E8e_00_2e_01_" in saved[0]
    data = np.loadtxt(tmp_path / saved[0], comments="#")
    rows, grids, st = R.run_mev_bands(_OracleContext(E, s), None, pixels=4)
    assert [r["E_min_MeV"] for r in rows] == [3.0, 8.0, 20.0] and st["rays"] == 48
    assert rows[1]["integrated_I_mev"] == pytest.approx(float(np.sum(data[:, 10])), rel=1e-12, abs=0.0)
    assert rows[1]["integrated_I_mev"] > 0.0
    for line in data:   # load_grid: grid[ny - 1 - j, i] = I_obs_mev
        assert grids[1][3 - int(line[1]), int(line[0])] == pytest.approx(line[10], rel=1e-8, abs=1e-300)
    csv_path, ppm = R.write_mev_bands(rows, grids, tmp_path / "bands")
    text = csv_path.read_text().splitlines()
    assert text[5] == "band,false_color,E_min_MeV,E_max_MeV,integrated_I_mev,data_path"
    assert text[7].startswith("intermediate-energy MeV band,green,8,20,")
    raw = ppm.read_bytes()
    assert raw.startswith(b"P6\n4 4\n255\n") and len(raw) == len(b"P6\n4 4\n255\n") + 4 * 4 * 3
