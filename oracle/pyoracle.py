"""ctypes access to the CPU ORACLE — test infrastructure only.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker (never by the product):
  * oracle_image(): the C restatement in oracle/hadros_oracle.c
    (oracle/liboracle.so, built by `make -C oracle`);
  * ref_image(): the reference itself, compiled from its own sources by
    oracle/build_ref.sh into oracle/_ref/libhadros_ref.so (present only where
    the reference sources were available at build time).
Both take the hadros_params struct of include/hadros_b200.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libhadros_ref.so"

_ORACLE = None
_REF = None


def build_oracle() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return ORACLE_SO


def oracle_lib() -> C.CDLL:
    global _ORACLE
    if _ORACLE is None:
        if not ORACLE_SO.exists():
            build_oracle()
        L = C.CDLL(str(ORACLE_SO))
        vp, i32 = C.c_void_p, C.c_int32
        L.hor_image.restype = C.c_int
        L.hor_image.argtypes = [vp, vp, vp, C.c_int, vp, i32] + [vp] * 13 + [C.c_int]
        L.hor_inverse_metric5.argtypes = [C.c_double, C.c_double, C.c_double, vp]
        L.hor_metric5.argtypes = [C.c_double, C.c_double, C.c_double, vp]
        L.hor_lapse.restype = C.c_double
        L.hor_lapse.argtypes = [C.c_double, C.c_double, C.c_double]
        L.hor_omega.restype = C.c_double
        L.hor_omega.argtypes = [C.c_double, C.c_double, C.c_double]
        L.hor_rho_params.restype = C.c_double
        L.hor_rho_params.argtypes = [vp, C.c_double, C.c_double]
        L.hor_rkf45_step.restype = C.c_int
        L.hor_rkf45_step.argtypes = [C.c_double, C.c_double, C.c_double, vp]
        L.hor_sigma_interp.restype = C.c_double
        L.hor_sigma_interp.argtypes = [vp, vp, C.c_int, C.c_double]
        L.hor_trace_points.restype = C.c_int
        L.hor_trace_points.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp]
        _ORACLE = L
    return _ORACLE


def ref_available() -> bool:
    return REF_SO.exists()


def reference_root() -> Path | None:
    """The reference source tree: $HADROS_REFERENCE_ROOT, else the tree
    oracle/build_ref.sh built oracle/_ref from; None where neither exists."""
    cand = os.environ.get("HADROS_REFERENCE_ROOT")
    if not cand and (HERE / "_ref" / "REFERENCE_ROOT").exists():
        cand = (HERE / "_ref" / "REFERENCE_ROOT").read_text().strip()
    return Path(cand) if cand and Path(cand).is_dir() else None


def ref_lib() -> C.CDLL:
    global _REF
    if _REF is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (oracle/build_ref.sh needs the reference sources)")
        L = C.CDLL(str(REF_SO))
        vp, i32 = C.c_void_p, C.c_int32
        L.ref_image.restype = C.c_int
        L.ref_image.argtypes = [vp, C.c_char_p, vp, i32] + [vp] * 12 + [C.c_int]
        _REF = L
    return _REF


def _n_bins(p) -> int:
    return 1 if p.spectral_kind == 0 else max(int(p.n_bins), 1)


MEV_KEYS = ("tau_mev", "P_surv_mev", "I_obs_mev", "r_nu", "leakage")


def _alloc(P: int, B: int, mev: bool = False) -> dict:
    out = {"tau": np.zeros(P), "P_surv": np.zeros(P), "I_obs": np.zeros(P),
           "fate": np.zeros(P, np.int8), "steps": np.zeros(P, np.int32),
           "attempts": np.zeros(P, np.int32), "tau_E": np.zeros((P, B)), "I_E": np.zeros((P, B))}
    if mev:
        out.update({k: np.zeros(P) for k in MEV_KEYS})
    return out


def _mev_ptrs(out: dict) -> list:
    return [out[k].ctypes.data if k in out else None for k in MEV_KEYS]


def oracle_image(p, sig_E, sig_cm2, pixel_ids=None, threads: int = 0, mev: bool = False) -> dict:
    """The C restatement over a whole image or a pixel list (OpenMP); with
    mev=True also the MeV channel's five outputs."""
    L = oracle_lib()
    E = np.ascontiguousarray(sig_E, dtype=np.float64)
    S = np.ascontiguousarray(sig_cm2, dtype=np.float64)
    ids = None if pixel_ids is None else np.ascontiguousarray(pixel_ids, dtype=np.int32)
    P = int(p.nx) * int(p.ny) if ids is None else int(ids.size)
    B = _n_bins(p)
    out = _alloc(P, B, mev)
    rc = L.hor_image(C.addressof(p), E.ctypes.data, S.ctypes.data, int(E.size),
                     None if ids is None else ids.ctypes.data, 0 if ids is None else int(ids.size),
                     *(out[k].ctypes.data for k in ("tau", "P_surv", "I_obs", "fate", "steps",
                                                     "attempts", "tau_E", "I_E")),
                     *_mev_ptrs(out), int(threads))
    if rc < 0:
        raise RuntimeError(f"oracle hor_image failed ({rc})")
    return out


def ref_image(p, sig_E, sig_gev2, sig_cm2, pixel_ids=None, threads: int = 0,
              per_bin: bool = True, mev: bool = False) -> dict:
    """The reference's own code (KerrCamera::trace_pixel + integrate_kerr_ray_spectral).
    per_bin=False skips the extra per-bin integrate_kerr_ray calls (timing runs);
    mev=True returns the MeV channel's five outputs too."""
    from hadros_b200.workloads import write_sigma_file
    L = ref_lib()
    ids = None if pixel_ids is None else np.ascontiguousarray(pixel_ids, dtype=np.int32)
    P = int(p.nx) * int(p.ny) if ids is None else int(ids.size)
    B = _n_bins(p)
    out = _alloc(P, B, mev)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "sigma.dat")
        write_sigma_file(path, sig_E, sig_gev2, sig_cm2)
        rc = L.ref_image(C.addressof(p), path.encode(), None if ids is None else ids.ctypes.data,
                         0 if ids is None else int(ids.size),
                         *(out[k].ctypes.data for k in ("tau", "P_surv", "I_obs", "fate", "steps")),
                         out["tau_E"].ctypes.data if per_bin else None,
                         out["I_E"].ctypes.data if per_bin else None,
                         *_mev_ptrs(out), int(threads))
    if rc < 0:
        raise RuntimeError(f"reference ref_image failed ({rc})")
    del out["attempts"]
    return out
