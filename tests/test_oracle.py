"""The CPU oracle against the reference: golden fixtures made by the
reference itself, the reference's own printed metric values, and (where the
reference was built here) the reference live."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

from conftest import golden_names, load_golden
from oracle import pyoracle as O

FIELDS = ("tau", "P_surv", "I_obs", "fate", "steps", "tau_E", "I_E")
# the heavy cases are covered by the GPU tests and the live reference test
CPU_CASES = [n for n in golden_names(near_ties=True) if n not in ("plain_tracer_32", "mixed_cfg_16_fp64")]


@pytest.mark.parametrize("name", CPU_CASES)
def test_oracle_bit_exact_vs_reference_fixture(hb, sigma_arrays, name):
    kw, ref = load_golden(name)
    E, _, s = sigma_arrays
    got = O.oracle_image(hb.params(**kw), E, s, pixel_ids=ref.get("pixel_ids"))
    for k in FIELDS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=f"{name}: {k}")


MEV_CASES = [n for n in CPU_CASES if n.startswith("mev_")]


@pytest.mark.parametrize("name", MEV_CASES)
def test_oracle_mev_channel_bit_exact_vs_reference_fixture(hb, sigma_arrays, name):
    """The MeV thermal channel (radiative_transfer.cpp:522-638 with
    mev_neutrino_physics.cpp) of the C restatement equals the reference's."""
    kw, ref = load_golden(name)
    E, _, s = sigma_arrays
    got = O.oracle_image(hb.params(**kw), E, s, mev=True)
    for k in FIELDS + O.MEV_KEYS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=f"{name}: {k}")


def test_mev_fixtures_exercise_the_channel():
    """The MeV fixtures are not trivial: optically thick and thin rays,
    neutrinospheres found and not, defaults for the empty band."""
    _, thick = load_golden("mev_physical_collapsar")
    assert thick["tau_mev"].max() > 1.0 and (thick["r_nu"] > 0).any()
    assert (thick["I_obs_mev"] > 0).all()
    _, thin = load_golden("mev_gaussian_thin")
    assert (thin["r_nu"] < 0).any()
    _, empty = load_golden("mev_empty_band")
    np.testing.assert_array_equal(empty["tau_mev"], 0.0)
    np.testing.assert_array_equal(empty["r_nu"], -1.0)
    np.testing.assert_array_equal(empty["leakage"], 1.0)


def test_oracle_bit_exact_plain_tracer_subset(hb, sigma_arrays):
    """Every 5th pixel of the 32x32 plain tracer (the full image is in the GPU tests)."""
    kw, ref = load_golden("plain_tracer_32")
    E, _, s = sigma_arrays
    ids = np.arange(0, 1024, 5, dtype=np.int32)
    got = O.oracle_image(hb.params(**kw), E, s, pixel_ids=ids)
    for k in FIELDS:
        np.testing.assert_array_equal(got[k], ref[k][ids], err_msg=k)


def test_known_answers_test_kerr_metric(hb):
    """apps/test_kerr_metric.cpp prints g, g^-1, lapse and omega at a=0.9, r=5,
    theta=pi/2 (printed with 8 significant digits)."""
    L = O.oracle_lib()
    g = np.zeros(5)
    gi = np.zeros(5)
    L.hor_metric5(0.9, 5.0, math.pi / 2.0, g.ctypes.data)
    L.hor_inverse_metric5(0.9, 5.0, math.pi / 2.0, gi.ctypes.data)
    expect_g = {"tph": -3.6e-01, "rr": 1.58127767, "thth": 25.0, "phph": 26.134}
    expect_gi = {"tt": -1.65300443, "tph": -2.27703985e-02, "rr": 0.6324, "thth": 0.04,
                 "phph": 3.79506641e-02}
    idx = {"tt": 0, "tph": 1, "rr": 2, "thth": 3, "phph": 4}
    for k, v in expect_g.items():
        assert g[idx[k]] == pytest.approx(v, rel=1e-8), k
    for k, v in expect_gi.items():
        assert gi[idx[k]] == pytest.approx(v, rel=1e-8), k
    assert L.hor_lapse(0.9, 5.0, math.pi / 2.0) == pytest.approx(0.77779114, rel=1e-8)
    assert L.hor_omega(0.9, 5.0, math.pi / 2.0) == pytest.approx(1.37751588e-02, rel=1e-8)
    # horizon radius r_+ = 1 + sqrt(1 - a^2)
    assert 1.0 + math.sqrt(1.0 - 0.81) == pytest.approx(1.43588989, rel=1e-8)


def test_oracle_sigma_interp_matches_library(hb, sigma_table, sigma_arrays):
    E, _, s = sigma_arrays
    L = O.oracle_lib()
    rng = np.random.default_rng(7)
    xs = np.concatenate([E[:3], E[-3:], 10.0 ** rng.uniform(4.0, 12.0, 200)])
    for x in xs:
        a = L.hor_sigma_interp(E.ctypes.data, s.ctypes.data, int(E.size), float(x))
        assert a == sigma_table.sigma_cm2(float(x))


def test_step_cap_truncates_prefix(hb, sigma_arrays):
    """A smaller cap keeps the first N steps of the uncapped ray (the rule the
    reference driver applies, src/kerr_camera.cpp:222)."""
    from hadros_b200 import workloads as W
    E, _, s = sigma_arrays
    kw = W.mixed_512(nx=3, ny=3, precision="fp64", h=0.05)
    full = O.oracle_image(hb.params(**kw), E, s)
    cap = int(full["steps"].min()) - 7
    capped = O.oracle_image(hb.params(**dict(kw, max_steps=cap)), E, s)
    assert np.all(capped["steps"] == cap)
    assert np.all(capped["fate"] == 2)


@pytest.mark.skipif(not O.ref_available(), reason="reference not built here (oracle/build_ref.sh)")
def test_oracle_vs_reference_live_random(hb, sigma_arrays):
    """Seeded random small cameras: oracle restatement == reference, bit for bit."""
    from hadros_b200 import workloads as W
    E, g2, s = sigma_arrays
    rng = np.random.default_rng(11)
    for k in range(6):
        kw = W.mixed_512(nx=3, ny=2, precision="fp64", h=float(rng.uniform(0.03, 0.08)),
                         a_spin=float(rng.uniform(0.0, 0.998)),
                         theta_obs_deg=float(rng.uniform(5.0, 85.0)),
                         profile=int(rng.integers(0, 8)), source=int(rng.integers(0, 5)),
                         spectral=int(rng.integers(0, 3)), n_bins=int(rng.integers(1, 6)),
                         rho0_gcm3=float(10.0 ** rng.uniform(8, 12)))
        p = hb.params(**kw)
        a = O.oracle_image(p, E, s)
        b = O.ref_image(p, E, g2, s)
        for f in FIELDS:
            np.testing.assert_array_equal(a[f], b[f], err_msg=f"case {k}: {f}")


@pytest.mark.skipif(not O.ref_available(), reason="reference not built here (oracle/build_ref.sh)")
def test_oracle_mev_channel_vs_reference_live_random(hb, sigma_arrays):
    """Seeded random MeV settings (model, flavor, profiles, band, switches,
    temperatures and Ye bounds) on random small cameras: the oracle's MeV
    channel == the reference's, bit for bit."""
    from hadros_b200 import workloads as W
    E, g2, s = sigma_arrays
    rng = np.random.default_rng(23)
    names = dict(mev_thermal=["constant", "inner_hot_torus", "radial_powerlaw", "torus_plus_cool_envelope",
                              "collapsar_inner_hot"],
                 mev_ye=["constant", "neutron_rich_torus", "funnel_proton_rich", "torus_envelope_contrast",
                         "collapsar_neutron_rich"],
                 mev_flavor=["nu_e", "anti_nu_e", "nu_x"], mev_model=["toy", "physical"],
                 mev_spectral=["monochromatic", "fermi_dirac_band"])
    switches = ["urca", "pair", "brems", "absorption", "scattering", "degeneracy_correction", "abs_n", "abs_p",
                "scat_n", "scat_p", "scat_e"]
    for k in range(8):
        kw = W.mixed_512(nx=3, ny=2, precision="fp64", h=float(rng.uniform(0.03, 0.08)),
                         a_spin=float(rng.uniform(0.0, 0.998)), theta_obs_deg=float(rng.uniform(5.0, 85.0)),
                         profile=int(rng.integers(0, 8)), source=int(rng.integers(0, 5)),
                         spectral=int(rng.integers(0, 3)), n_bins=int(rng.integers(1, 6)),
                         rho0_gcm3=float(10.0 ** rng.uniform(8, 12)), mev_channel=1,
                         mev_n_bins=int(rng.integers(1, 7)), mev_T0_MeV=float(rng.uniform(1.0, 15.0)),
                         mev_T_floor_MeV=float(rng.uniform(0.01, 0.5)), mev_T_power=float(rng.uniform(0.0, 1.0)),
                         mev_Ye_floor=float(rng.uniform(0.0, 0.2)), mev_Ye_ceil=float(rng.uniform(0.4, 1.0)),
                         mev_Enu_obs_MeV=float(rng.uniform(3.0, 40.0)),
                         mev_E_min_MeV=float(rng.uniform(1.0, 5.0)), mev_E_max_MeV=float(rng.uniform(20.0, 80.0)),
                         **{key: str(rng.choice(v)) for key, v in names.items()},
                         **{f"mev_{sw}": bool(rng.integers(0, 2)) for sw in switches})
        p = hb.params(**kw)
        a = O.oracle_image(p, E, s, mev=True)
        b = O.ref_image(p, E, g2, s, mev=True)
        for f in O.MEV_KEYS:
            np.testing.assert_array_equal(a[f], b[f], err_msg=f"case {k}: {f}")
