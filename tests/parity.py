"""Comparison rules of the parity tests.

FP64 mode: fate and accepted-step count equal per pixel; tau, P_surv and I
within 1e-6 relative.  Mixed mode (FP32 Kahan transfer): fate and steps
equal; tau and I within 1e-4 relative, and P_surv = exp(-tau) within 1e-4
absolute (an error of 1e-4*tau in tau moves exp(-tau) by at most 3.7e-5).  Intensities far below the image's
brightest pixel carry no information in either arithmetic, so I is compared
with an absolute floor of 1e-30 * max|I| (and 1e-290: subnormal values).
The MeV channel is FP64 in both modes: its five outputs (where both sides
have them) are held to 1e-6 relative, its intensity with the same floor.
"""
from __future__ import annotations

import numpy as np

RTOL_FP64 = 1.0e-6
MEV_KEYS = ("tau_mev", "P_surv_mev", "I_obs_mev", "r_nu", "leakage")
RTOL_MIXED = 1.0e-4
I_FLOOR = 1.0e-30
# intensities below this are FP64 subnormal/underflow noise in both paths
I_ABS_FLOOR = 1.0e-290


def rel_err(got, ref, floor=0.0):
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.maximum(np.abs(ref), floor)
    with np.errstate(invalid="ignore", divide="ignore"):
        e = np.where(den > 0, np.abs(got - ref) / np.where(den > 0, den, 1.0), np.abs(got - ref))
    return e


def assert_parity(got: dict, ref: dict, rtol: float, label: str = "", p_absolute: bool = False) -> dict:
    np.testing.assert_array_equal(got["fate"], ref["fate"], err_msg=f"{label}: ray fate")
    np.testing.assert_array_equal(got["steps"], ref["steps"], err_msg=f"{label}: accepted steps")
    imax = float(np.max(np.abs(ref["I_obs"]))) if ref["I_obs"].size else 0.0
    errs = {
        "tau": float(np.max(rel_err(got["tau"], ref["tau"]), initial=0.0)),
        "P_surv": float(np.max(rel_err(got["P_surv"], ref["P_surv"], 1.0 if p_absolute else 1e-300),
                               initial=0.0)),
        "I_obs": float(np.max(rel_err(got["I_obs"], ref["I_obs"], max(I_FLOOR * imax, I_ABS_FLOOR)),
                              initial=0.0)),
    }
    if "tau_E" in got and "tau_E" in ref:
        iemax = float(np.max(np.abs(ref["I_E"]))) if ref["I_E"].size else 0.0
        errs["tau_E"] = float(np.max(rel_err(got["tau_E"], ref["tau_E"]), initial=0.0))
        errs["I_E"] = float(np.max(rel_err(got["I_E"], ref["I_E"], max(I_FLOOR * iemax, I_ABS_FLOOR)),
                                   initial=0.0))
    for k, v in errs.items():
        assert v <= rtol, f"{label}: {k} relative error {v:.3e} > {rtol:.1e}"
    if all(k in got and k in ref for k in MEV_KEYS):
        errs.update(mev_errors(got, ref))
        for k in MEV_KEYS:
            assert errs[k] <= RTOL_FP64, f"{label}: {k} relative error {errs[k]:.3e} > {RTOL_FP64:.1e}"
    return errs


def mev_errors(got: dict, ref: dict) -> dict:
    """Largest relative error of each MeV channel output."""
    mmax = float(np.max(np.abs(ref["I_obs_mev"]))) if ref["I_obs_mev"].size else 0.0
    floors = {"tau_mev": 0.0, "P_surv_mev": 1e-300, "I_obs_mev": max(I_FLOOR * mmax, I_ABS_FLOOR),
              "r_nu": 0.0, "leakage": 0.0}
    return {k: float(np.max(rel_err(got[k], ref[k], floors[k]), initial=0.0)) for k in MEV_KEYS}
