"""The reference's image files: names, 13-column text image and KIMG binary,
written by the library from host arrays (no GPU)."""
from __future__ import annotations

import ctypes as C
import struct
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, load_golden


def fname(hb, p, style, ext, dis=None, mev_E=10.0, mev_norm=1.0):
    buf = C.create_string_buffer(512)
    rc = hb.lib().hadros_image_filename(C.byref(p), style, dis, mev_E, mev_norm, ext.encode(), buf, 512)
    assert rc == 0
    return buf.value.decode()


def test_filenames_match_reference_validation_targets(hb):
    """Names the reference Makefile's validate_small_cuda target compares
    (Makefile:686-687: ENU 1e5, TORUS_RHO0 1e-2, CAM_THETA_DEG 80, MeV 10/1)."""
    p = hb.params(Enu_obs_GeV=1e5, rho0_gcm3=1e-2, theta_obs_deg=80.0)
    assert fname(hb, p, 1, ".dat", b"GBW") == (
        "kerr_image_cuda_cache_GBW_rho0_torus_1e-2_Enu_1e_05_MeVEnu_1e_01_MeVNorm_1e_00_CamTheta_80p0.dat")
    q = hb.params(Enu_obs_GeV=1e5, rho0_gcm3=1e-2, theta_obs_deg=80.0, profile="powerlaw_funnel_envelope")
    assert fname(hb, q, 1, ".dat", b"GBW") == (
        "kerr_image_cuda_cache_GBW_rho0_torus_1e-2_Profile_powerlaw_funnel_envelope_Enu_1e_05_"
        "MeVEnu_1e_01_MeVNorm_1e_00_CamTheta_80p0.dat")
    r = hb.params(Enu_obs_GeV=1e9, rho0_gcm3=1e11, theta_obs_deg=17.0, source="funnel_wall",
                  spectral="powerlaw_cutoff")
    assert fname(hb, r, 0, ".bin") == (
        "kerr_image_cuda_rho0_torus_1e11_Source_funnel_wall_Enu_1e_09_MeVEnu_1e_01_MeVNorm_1e_00_"
        "CamTheta_17p0.bin")
    assert fname(hb, r, 1, ".dat", b"IIM") == (
        "kerr_image_cuda_cache_IIM_rho0_torus_1e11_Source_funnel_wall_Spectrum_powerlaw_cutoff_"
        "Enu_1e_09_MeVEnu_1e_01_MeVNorm_1e_00_CamTheta_17p0.dat")


def _write(hb, tmp_path, kw, ref):
    p = hb.params(**kw)
    arrs = [np.ascontiguousarray(ref[k]) for k in ("tau", "P_surv", "I_obs", "fate")]
    dat, kimg = tmp_path / "img.dat", tmp_path / "img.bin"
    L = hb.lib()
    assert L.hadros_write_dat(str(dat).encode(), C.byref(p), b"GBW", 10.0, 1.0,
                              *(a.ctypes.data for a in arrs)) == 0
    assert L.hadros_write_kimg(str(kimg).encode(), C.byref(p), 10.0, 1.0,
                               *(a.ctypes.data for a in arrs)) == 0
    return p, dat, kimg


def test_dat_and_kimg_layout(hb, tmp_path):
    kw, ref = load_golden("edge_ragged_3x5")
    p, dat, kimg = _write(hb, tmp_path, kw, ref)
    text = dat.read_text().splitlines()
    assert text[0] == "# profile_type powerlaw_funnel_envelope"
    assert "# source_model funnel_wall" in text
    assert "# spectral_model powerlaw_cutoff" in text
    assert text[[i for i, l in enumerate(text) if not l.startswith("#")][0] - 1].startswith(
        "# i j alpha beta tau_uhe P_surv_uhe I_obs_uhe captured")
    d = np.loadtxt(dat, comments="#")
    assert d.shape == (15, 13)
    np.testing.assert_array_equal(d[:, 0], np.tile(np.arange(3), 5))
    np.testing.assert_array_equal(d[:, 1], np.repeat(np.arange(5), 3))
    np.testing.assert_allclose(d[:, 4], ref["tau"], rtol=1e-8)
    np.testing.assert_allclose(d[:, 6], ref["I_obs"], rtol=1e-8)
    np.testing.assert_array_equal(d[:, 7], (ref["fate"] == 1).astype(float))
    np.testing.assert_array_equal(d[:, 8:], np.tile([0.0, 1.0, 0.0, -1.0, 1.0], (15, 1)))
    with open(kimg, "rb") as f:
        h = struct.Struct("<7i4d")
        magic, version, backend, nx, ny, ncols, res, E, Emev, norm, th = h.unpack(f.read(h.size))
        payload = np.fromfile(f, dtype="<f8")
    assert (magic, version, nx, ny, ncols) == (0x4B494D47, 1, 3, 5, 13)
    assert th == pytest.approx(17.0)
    rows = payload.reshape(15, 13)
    np.testing.assert_array_equal(rows[:, 4], ref["tau"])
    np.testing.assert_array_equal(rows[:, 6], ref["I_obs"])
    np.testing.assert_allclose(rows[:, :4], d[:, :4], rtol=1e-8)


def test_mev_columns_and_header(hb, tmp_path):
    """hadros_write_dat_mev / hadros_write_kimg_mev: the MeV channel's five
    columns and, with the channel on, the CPU app's MeV metadata lines."""
    kw, ref = load_golden("mev_fd_band_spectral")
    p = hb.params(**kw)
    host = {k: np.ascontiguousarray(ref[k]) for k in ("tau", "P_surv", "I_obs", "fate") + hb.MEV_OUTPUTS}
    out = hb.HadrosImageOut()
    for k, a in host.items():
        setattr(out, k, a.ctypes.data)
    dat, kimg = tmp_path / "m.dat", tmp_path / "m.bin"
    L = hb.lib()
    assert L.hadros_write_dat_mev(str(dat).encode(), C.byref(p), b"GBW", C.byref(out)) == 0
    assert L.hadros_write_kimg_mev(str(kimg).encode(), C.byref(p), C.byref(out)) == 0
    text = dat.read_text().splitlines()
    for line in ("# MEV_MODEL physical", "# MEV_FLAVOR anti_nu_e", "# MEV_THERMAL_PROFILE inner_hot_torus",
                 "# MEV_YE_PROFILE neutron_rich_torus", "# MEV_SPECTRAL_MODE fermi_dirac_band",
                 "# MEV_N_BINS 5", "# MEV_INCLUDE_URCA 1", "# MEV_USE_DEGENERACY_CORRECTION 0",
                 "# mev_opacity_units cm^-1"):
        assert line in text, line
    d = np.loadtxt(dat, comments="#")
    for c, k in enumerate(hb.MEV_OUTPUTS):
        np.testing.assert_allclose(d[:, 8 + c], ref[k], rtol=1e-8, err_msg=k)
    rows = np.fromfile(kimg, dtype="<f8", offset=struct.calcsize("<7i4d")).reshape(-1, 13)
    for c, k in enumerate(hb.MEV_OUTPUTS):
        np.testing.assert_array_equal(rows[:, 8 + c], ref[k], err_msg=k)
    # the CPU app's file name carries the MeV band
    assert "_MeVSpectrum_fermi_dirac_band_E3e_00_5e_01_" in fname(hb, p, 1, ".dat", b"GBW")
    # a missing array writes its default
    out.r_nu = None
    assert L.hadros_write_dat_mev(str(dat).encode(), C.byref(p), b"GBW", C.byref(out)) == 0
    np.testing.assert_array_equal(np.loadtxt(dat, comments="#")[:, 11], -1.0)


def test_mev_names_and_validation(hb):
    L = hb.lib()
    k = C.c_int32()
    for fn, name, want in (("hadros_parse_mev_model", b"phys", 1), ("hadros_parse_mev_flavor", b"anti-nu-e", 1),
                           ("hadros_parse_mev_thermal", b"COLLAPSAR_INNER_HOT", 4),
                           ("hadros_parse_mev_ye", b"funnel_proton_rich", 2),
                           ("hadros_parse_mev_spectral", b"fd_band", 1)):
        assert getattr(L, fn)(name, C.byref(k)) == 0 and k.value == want
    assert L.hadros_parse_mev_flavor(b"nu_tau", C.byref(k)) == hb.abi.E_ARG
    assert L.hadros_last_error().decode() == "Unknown MEV_FLAVOR 'nu_tau'. Use nu_e, anti_nu_e, or nu_x."
    assert L.hadros_mev_thermal_name(3) == b"torus_plus_cool_envelope"
    assert L.hadros_mev_ye_name(9) is None
    p = hb.params(mev_channel=1)
    assert L.hadros_params_validate(C.byref(p)) == 0
    p.mev_flavor = 3
    assert L.hadros_params_validate(C.byref(p)) == hb.abi.E_ARG
    p.mev_channel = 0   # the channel's fields are ignored while it is off
    assert L.hadros_params_validate(C.byref(p)) == 0
    q = hb.params(mev_channel=1, mev_T0_MeV=float("nan"))
    assert L.hadros_params_validate(C.byref(q)) == hb.abi.E_ARG
    d = hb.params()
    assert (d.mev_channel, d.mev_model, d.mev_flavor, d.mev_flags) == (0, 1, 1, 0x7DF)
    assert d.mev_neutrinosphere_tau == 2.0 / 3.0 and d.mev_sigma_abs0_cm2 == 9.6e-44


def test_alpha_beta_are_reference_camera_coordinates(hb, tmp_path):
    import math
    kw, ref = load_golden("edge_ragged_3x5")
    p, dat, kimg = _write(hb, tmp_path, kw, ref)
    rows = np.fromfile(kimg, dtype="<f8", offset=struct.calcsize("<7i4d")).reshape(15, 13)
    t = math.tan(0.5 * (p.fov_deg * math.pi / 180.0))
    for row in rows:
        i, j = int(row[0]), int(row[1])
        assert row[2] == (2.0 * (i + 0.5) / p.nx - 1.0) * t
        assert row[3] == (2.0 * (j + 0.5) / p.ny - 1.0) * t


def test_compare_module_matches_reference_script(hb, tmp_path):
    """hadros_b200.compare's aggregates equal the reference comparer's."""
    from oracle import pyoracle as O
    root = O.reference_root()
    script = (root / "scripts" / "compare_cuda_cpu_metrics.py") if root else Path("/nonexistent")
    kw, ref = load_golden("edge_ragged_3x5")
    _, dat_a, _ = _write(hb, tmp_path, kw, ref)
    ref2 = dict(ref)
    ref2["tau"] = ref["tau"] * (1 + 1e-7)
    d2 = tmp_path / "b"
    d2.mkdir()
    _, dat_b, _ = _write(hb, d2, kw, ref2)
    ours = tmp_path / "ours.txt"
    from hadros_b200 import compare
    assert compare.main([str(ours), "case", str(dat_a), str(dat_b)]) == 0
    got = {l.split()[0]: l.split()[1:] for l in ours.read_text().splitlines()
           if l and not l.startswith(("#", "[", "cpu_", "gpu_", "per_"))}
    assert float(got["mean_tau"][2]) == pytest.approx(1e-7, rel=1e-2)
    if not script.exists():
        pytest.skip("reference comparer not present here")
    theirs = tmp_path / "theirs.txt"
    subprocess.run([sys.executable, str(script), str(theirs), "case", str(dat_a), str(dat_b)],
                   check=True, capture_output=True)
    ref_m = {l.split()[0]: l.split()[1:] for l in theirs.read_text().splitlines()
             if l and not l.startswith(("#", "[", "cpu_", "cuda_"))}
    for k in ("mean_tau", "max_tau", "mean_P_surv", "total_intensity", "valid_rays"):
        assert got[k] == ref_m[k], k


def test_cli_usage_and_errors():
    cli = ROOT / "hadros_b200" / "bin" / "compute_kerr_image"
    if not cli.exists():
        pytest.skip("CLI not built")
    r = subprocess.run([str(cli), "1e9", "0.9", "3", "1e-2", "10", "5", "0.25", "3.5", "1", "15", "2",
                        "1e12", "1", "10", "1", "80", "60", "25", "0", "10"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr
    r = subprocess.run([str(cli), "--sigma=/nonexistent.dat"], capture_output=True, text=True)
    assert r.returncode == 1 and "Could not open sigma table" in r.stderr
    r = subprocess.run([str(cli), "1e9", "0.9", "3", "1e-2", "10", "5", "0.25", "3.5", "1", "15", "2",
                        "1e12", "1", "10", "1", "80", "60", "25", "4", "4", "120", "0.01", "32", "128",
                        "200000", "1e-6", "no_such_profile"], capture_output=True, text=True)
    assert r.returncode == 1 and "Unknown density profile 'no_such_profile'" in r.stderr


def test_cli_cache_modes_usage_and_errors(tmp_path):
    """--geodesic-cache and --image-from-cache (the reference executable's
    cache modes) reject what the reference rejects, before any GPU work."""
    cli = ROOT / "hadros_b200" / "bin" / "compute_kerr_image"
    if not cli.exists():
        pytest.skip("CLI not built")
    r = subprocess.run([str(cli), "--geodesic-cache", "0.9", "60", "80", "25", "0", "4"], capture_output=True,
                       text=True, cwd=tmp_path)
    assert r.returncode == 1 and "--geodesic-cache ASPIN CAM_R_OBS" in r.stderr
    r = subprocess.run([str(cli), "--image-from-cache", "1e9", "0.9", "3", "1e-2", "10", "5", "0.25", "3.5", "1",
                        "15", "2", "1e12", "1", "10", "1", "80", "0"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 1 and "--image-from-cache ENU ASPIN" in r.stderr
    r = subprocess.run([str(cli), "--image-from-cache", "1e9"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 1 and "output/rays/kerr_geodesics_cuda.bin" in r.stderr
    r = subprocess.run([str(cli), "--image-from-cache", "1e9", "--mev=bogus"], capture_output=True, text=True,
                       cwd=tmp_path)
    assert r.returncode == 1 and "Unknown MEV_MODEL 'bogus'" in r.stderr

