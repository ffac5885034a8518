"""KGEO geodesic cache files: round trip, error behaviour, and compatibility
with the reference's own cache writer and reader (built from its sources into
oracle/_ref by oracle/build_ref.sh; those tests skip where it is absent)."""
from __future__ import annotations

import ctypes as C
import math
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import pyoracle as O

REF_DIR = Path(O.__file__).resolve().parent / "_ref"
REF_GEO = REF_DIR / "compute_kerr_geodesics"
REF_IMG = REF_DIR / "compute_kerr_image_from_cache"


def oracle_paths(hb, p, E, s):
    """Per-pixel PathPoints from the oracle: (r, theta, x, y, z, dl, redshift)."""
    L = O.oracle_lib()
    n_all, pts_all, fates = [], [], []
    for pid in range(p.nx * p.ny):
        i, j = pid % p.nx, pid // p.nx
        buf = np.zeros((250000, 5))
        n, f = C.c_int32(), C.c_int32()
        cnt = L.hor_trace_points(C.addressof(p), E.ctypes.data, s.ctypes.data, int(E.size), i, j,
                                 250000, buf.ctypes.data, C.byref(n), C.byref(f))
        q = buf[:cnt]
        r, th, ph = q[:, 0], q[:, 1], q[:, 2]
        seven = np.stack([r, th, r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph),
                          r * np.cos(th), q[:, 3], q[:, 4]], axis=1)
        n_all.append(cnt)
        pts_all.append(seven)
        fates.append(f.value)
    return np.array(n_all, np.int32), np.concatenate(pts_all), np.array(fates, np.int8)


def test_kgeo_roundtrip(hb, tmp_path):
    p = hb.params(nx=3, ny=2, a_spin=0.7)
    n = np.array([2, 0, 3, 1, 0, 4], np.int32)
    pts = np.random.default_rng(1).normal(size=(int(n.sum()), 7))
    fate = np.array([1, 0, 0, 2, 1, 0], np.int8)
    f = tmp_path / "c.bin"
    hb.write_kgeo(f, p, n, pts, fate=fate)
    assert f.stat().st_size == 24 + 40 * 6 + 56 * int(n.sum())
    raw = f.read_bytes()
    assert struct.unpack("<4id", raw[:24]) == (0x4B47454F, 1, 3, 2, 0.7)
    ray_id, pi, pj, cap, npt = struct.unpack("<5i", raw[24:44])
    assert (ray_id, pi, pj, cap, npt) == (0, 0, 0, 1, 2)      # ray_id = i*ny + j
    d = hb.read_kgeo(f)
    assert (d["nx"], d["ny"], d["a_spin"]) == (3, 2, 0.7)
    np.testing.assert_array_equal(d["pixel_ids"], np.arange(6))
    np.testing.assert_array_equal(d["npoints"], n)
    np.testing.assert_array_equal(d["captured"], (fate == 1).astype(np.int8))
    np.testing.assert_array_equal(d["points"], pts)
    t = math.tan(0.5 * math.radians(p.fov_deg))
    assert d["alpha"][4] == (2.0 * (1 + 0.5) / 3 - 1.0) * t


def test_kgeo_written_in_batches_equals_one_write(hb, tmp_path):
    """hadros_write_kgeo_rays: a file written in three batches (header with
    the first) has the bytes of the single write."""
    p = hb.params(nx=3, ny=2, a_spin=0.7)
    n = np.array([2, 0, 3, 1, 0, 4], np.int32)
    pts = np.random.default_rng(2).normal(size=(int(n.sum()), 7))
    fate = np.array([1, 0, 0, 2, 1, 0], np.int8)
    one, parts = tmp_path / "one.bin", tmp_path / "parts.bin"
    hb.write_kgeo(one, p, n, pts, fate=fate)
    off = np.concatenate([[0], np.cumsum(n)])
    for b, (lo, hi) in enumerate(((0, 2), (2, 3), (3, 6))):
        hb.write_kgeo(parts, p, n[lo:hi], pts[off[lo]:off[hi]], pixel_ids=np.arange(lo, hi, dtype=np.int32),
                      fate=fate[lo:hi], append=b > 0)
    assert parts.read_bytes() == one.read_bytes()
    with pytest.raises(hb.HadrosError, match="No KGEO file to append to"):
        hb.write_kgeo(tmp_path / "missing.bin", p, n[:1], pts[:2], append=True)


def test_kgeo_errors(hb, tmp_path):
    p = hb.params(nx=2, ny=1)
    f = tmp_path / "c.bin"
    hb.write_kgeo(f, p, np.array([1, 2], np.int32), np.zeros((3, 7)))
    raw = bytearray(f.read_bytes())
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"XXXX" + raw[4:])
    with pytest.raises(hb.HadrosError, match="bad magic number"):
        hb.read_kgeo(bad)
    bad.write_bytes(raw[:4] + struct.pack("<i", 2) + raw[8:])
    with pytest.raises(hb.HadrosError, match="Unsupported binary geodesic cache version: 2"):
        hb.read_kgeo(bad)
    bad.write_bytes(raw[:-10])
    with pytest.raises(hb.HadrosError, match="Unexpected end of file"):
        hb.read_kgeo(bad)
    neg = raw[:24] + raw[24:40] + struct.pack("<i", -1) + raw[44:]
    bad.write_bytes(neg)
    with pytest.raises(hb.HadrosError, match="negative number of points"):
        hb.read_kgeo(bad)
    with pytest.raises(hb.HadrosError, match="Could not open"):
        hb.read_kgeo(tmp_path / "missing.bin")


def _fmt(x):
    return f"{x:.17g}"


@pytest.mark.skipif(not REF_IMG.exists(), reason="reference cache executables not built here")
def test_reference_reads_our_kgeo(hb, tmp_path, sigma_arrays):
    """Our KGEO, written from oracle paths, fed to the reference's own
    compute_kerr_image_from_cache: its image equals the oracle's."""
    from hadros_b200 import workloads as W
    E, g2, s = sigma_arrays
    kw = W.mixed_512(nx=4, ny=3, h=0.05, precision="fp64")
    p = hb.params(**kw)
    n, pts, fate = oracle_paths(hb, p, E, s)
    cache = tmp_path / "cache.bin"
    hb.write_kgeo(cache, p, n, pts, fate=fate)
    sig = tmp_path / "sigma.dat"
    W.write_sigma_file(sig, E, g2, s)
    (tmp_path / "output" / "images").mkdir(parents=True)
    argv = [str(REF_IMG), "1e9", _fmt(p.a_spin), _fmt(p.M_bh_msun), _fmt(p.rho0_gcm3), _fmt(p.r0_rg),
            _fmt(p.sigma_r_rg), _fmt(p.H_over_R), _fmt(p.src_r_center_rg), _fmt(p.src_sigma_r_rg),
            _fmt(kw["src_theta_width_deg"]), _fmt(p.src_powerlaw), _fmt(p.src_emax_GeV), _fmt(p.src_norm),
            "10", "1", _fmt(kw["theta_obs_deg"]), str(sig), "powerlaw_funnel_envelope",
            _fmt(p.radial_power), _fmt(p.funnel_depletion), _fmt(kw["funnel_theta_deg"]),
            _fmt(p.envelope_rho0_gcm3), _fmt(p.envelope_alpha), _fmt(p.torus_r_min_rg),
            _fmt(p.torus_r_max_rg), _fmt(p.rho_floor_gcm3), _fmt(p.r_obs_rg), "1", str(cache),
            "funnel_wall", _fmt(kw["src_funnel_theta_deg"]), _fmt(p.src_density_power_q),
            _fmt(p.src_radial_power_s), _fmt(p.src_gradient_dr_rg), "1", _fmt(p.src_rho_ref_gcm3),
            _fmt(p.src_cutoff_min), _fmt(p.src_cutoff_max), "powerlaw_cutoff", _fmt(p.spec_gamma),
            _fmt(p.spec_ecut_GeV), _fmt(p.spec_e_min_GeV), _fmt(p.spec_e_max_GeV), str(p.n_bins)]
    r = subprocess.run(argv, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    dat = next((tmp_path / "output" / "images").glob("*.dat"))
    buf = C.create_string_buffer(512)
    hb.lib().hadros_image_filename(C.byref(p), 1, b"GBW", 10.0, 1.0, b".dat", buf, 512)
    assert dat.name == buf.value.decode()          # the name the scan scripts re-derive
    d = np.loadtxt(dat, comments="#")
    ref = O.oracle_image(p, E, s)
    for row in d:
        k = int(row[1]) * p.nx + int(row[0])
        assert row[4] == pytest.approx(ref["tau"][k], rel=1e-8, abs=1e-300)
        assert row[6] == pytest.approx(ref["I_obs"][k], rel=1e-8, abs=1e-300)
        assert int(row[7]) == int(ref["fate"][k] == 1)


@pytest.mark.skipif(not REF_GEO.exists(), reason="reference cache executables not built here")
def test_we_read_reference_kgeo(hb, tmp_path, sigma_arrays):
    """The reference's compute_kerr_geodesics writes a cache (rays in
    OpenMP order); our reader recovers each pixel's points and fate."""
    E, _, s = sigma_arrays
    out = tmp_path / "geo.bin"
    args = ["0.8", "60", "40", "25", "3", "2", "120", "0.05", str(out)]
    r = subprocess.run([str(REF_GEO), *args], capture_output=True, text=True, timeout=300,
                       env={"OMP_NUM_THREADS": "2"})
    assert r.returncode == 0, r.stderr
    d = hb.read_kgeo(out)
    assert (d["nx"], d["ny"], d["a_spin"]) == (3, 2, 0.8)
    p = hb.params(a_spin=0.8, r_obs_rg=60.0, theta_obs_rad=math.pi * 40.0 / 180.0, fov_deg=25.0,
                  nx=3, ny=2, r_max_rg=120.0, h=0.05)
    ref = O.oracle_image(p, E, s)
    order = np.argsort(d["pixel_ids"])
    np.testing.assert_array_equal(d["pixel_ids"][order], np.arange(6))
    np.testing.assert_array_equal(d["npoints"][order], ref["steps"])
    np.testing.assert_array_equal(d["captured"][order], (ref["fate"] == 1).astype(np.int8))
    n, pts, _ = oracle_paths(hb, p, E, s)
    offs = np.concatenate([[0], np.cumsum(d["npoints"])])
    for k in range(6):
        pid = d["pixel_ids"][k]
        mine = pts[sum(n[:pid]):sum(n[:pid]) + n[pid]]
        theirs = d["points"][offs[k]:offs[k + 1]]
        np.testing.assert_array_equal(theirs[:, [0, 1, 5, 6]], mine[:, [0, 1, 5, 6]])
