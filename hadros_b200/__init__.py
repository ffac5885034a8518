"""hadros_b200 — B200-native HADROS per-pixel image pipeline.

Python face of the C ABI in include/hadros_b200.h (the library
hadros_b200/lib/libhadros_b200.so, built by ``python -m hadros_b200.build``).
The compute path is the CUDA library; there is no CPU fallback: without the
built library or a B200, the calls raise.

    import hadros_b200 as hb
    sig = hb.SigmaTable.load("data/sigma/sigma_nuN_CC_GBW.dat")
    p = hb.params(nx=32, ny=32, profile="gaussian", source="inner_ring")
    with hb.Context(0) as ctx:
        img = ctx.image(p, sig)          # dict of numpy arrays, pixel = j*nx + i
"""
from __future__ import annotations

import ctypes as C
import math
import os
from pathlib import Path

import numpy as np

from . import abi
from .abi import (FATE_CAPTURED, FATE_ESCAPED, FATE_TRUNCATED, ORDER_COST, ORDER_ROWS,
                  ORDER_TILES, PRECISION_FP64, PRECISION_MIXED, PROFILES, SOURCES, SPECTRA,
                  HadrosImageOut, HadrosParams, HadrosSchedule, HadrosStats)

__all__ = ["lib", "HadrosError", "params", "SigmaTable", "Context", "spectral_bins",
           "HadrosParams", "PRECISION_FP64", "PRECISION_MIXED", "PROFILES", "SOURCES",
           "SPECTRA", "FATE_ESCAPED", "FATE_CAPTURED", "FATE_TRUNCATED"]

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libhadros_b200.so"
_LIB = None


class HadrosError(RuntimeError):
    """A HADROS_E_* status from the library, with hadros_last_error()'s text."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status
        self.message = message


def lib() -> C.CDLL:
    """Load libhadros_b200.so (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        path = Path(os.environ.get("HADROS_B200_LIB", LIB_PATH))
        if not path.exists():
            raise ImportError(f"{path} not found: build it with `python -m hadros_b200.build`")
        L = C.CDLL(str(path))
        for name, (res, args) in abi.SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        if L.hadros_abi_version() != abi.ABI_VERSION:
            raise ImportError("libhadros_b200.so ABI version does not match hadros_b200/abi.py")
        _LIB = L
    return _LIB


def _check(status: int) -> None:
    if status != abi.OK:
        raise HadrosError(status, lib().hadros_last_error().decode())


def _kind(table, value, parser: str) -> int:
    if isinstance(value, str):
        k = C.c_int32()
        _check(getattr(lib(), parser)(value.encode(), C.byref(k)))
        return k.value
    return int(value)


_DEG = {"theta_obs_deg": "theta_obs_rad", "funnel_theta_deg": "funnel_theta_rad",
        "src_theta_width_deg": "src_theta_width_rad", "src_funnel_theta_deg": "src_funnel_theta_rad",
        "src_gradient_dtheta_deg": "src_gradient_dtheta_rad"}


# MeV channel names -> (parser, hadros_params field)
_MEV_NAMES = {"mev_model": ("hadros_parse_mev_model", "mev_model"),
              "mev_flavor": ("hadros_parse_mev_flavor", "mev_flavor"),
              "mev_thermal": ("hadros_parse_mev_thermal", "mev_thermal_profile"),
              "mev_ye": ("hadros_parse_mev_ye", "mev_ye_profile"),
              "mev_spectral": ("hadros_parse_mev_spectral", "mev_spectral_mode")}


def _mev_kind(fn: str, name: str) -> int:
    k = C.c_int32()
    _check(getattr(lib(), fn)(str(name).encode(), C.byref(k)))
    return k.value


def params(**kw) -> HadrosParams:
    """hadros_params_default() with overrides.

    Accepts every hadros_params field, the model names ``profile``, ``source``,
    ``spectral`` (reference spellings and aliases), ``precision`` as
    "fp64"/"mixed", and ``*_deg`` forms of the angle fields (converted as the
    reference apps do: value * M_PI / 180.0).  MeV channel: ``mev_channel``,
    the names ``mev_model``, ``mev_flavor``, ``mev_thermal``, ``mev_ye``,
    ``mev_spectral`` and one boolean per switch (``mev_urca``, ``mev_pair``,
    ``mev_brems``, ``mev_absorption``, ``mev_scattering``,
    ``mev_degeneracy_correction``, ``mev_abs_n``, ``mev_abs_p``, ``mev_scat_n``,
    ``mev_scat_p``, ``mev_scat_e``).
    """
    p = HadrosParams()
    lib().hadros_params_default(C.byref(p))
    for key, val in kw.items():
        if key == "profile":
            p.profile_kind = _kind(PROFILES, val, "hadros_parse_profile")
        elif key == "source":
            p.source_kind = _kind(SOURCES, val, "hadros_parse_source")
        elif key == "spectral":
            p.spectral_kind = _kind(SPECTRA, val, "hadros_parse_spectral")
        elif key == "fast":
            p.fast_geodesic = 1 if val else 0
        elif key == "precision":
            p.precision = {"fp64": PRECISION_FP64, "mixed": PRECISION_MIXED}.get(val, val)
        elif key in _MEV_NAMES:
            fn, field = _MEV_NAMES[key]
            setattr(p, field, val if isinstance(val, int) else _mev_kind(fn, val))
        elif key.startswith("mev_") and key[4:] in abi.MEV_FLAG_BITS:
            bit = abi.MEV_FLAG_BITS[key[4:]]
            p.mev_flags = (p.mev_flags | bit) if val else (p.mev_flags & ~bit)
        elif key in _DEG:
            setattr(p, _DEG[key], float(val) * math.pi / 180.0)
        elif hasattr(p, key):
            setattr(p, key, val)
        else:
            raise TypeError(f"unknown hadros_params field {key!r}")
    return p


class SigmaTable:
    """sigma_CC(E) table handle (SigmaTable, src/sigma_table.cpp)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    @classmethod
    def load(cls, path) -> "SigmaTable":
        h = C.c_void_p()
        _check(lib().hadros_sigma_load(str(path).encode(), C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_arrays(cls, E_GeV, sigma_cm2, sigma_GeV2=None) -> "SigmaTable":
        E = np.ascontiguousarray(E_GeV, dtype=np.float64)
        s = np.ascontiguousarray(sigma_cm2, dtype=np.float64)
        g = None if sigma_GeV2 is None else np.ascontiguousarray(sigma_GeV2, dtype=np.float64)
        if E.shape != s.shape or (g is not None and g.shape != E.shape):
            raise ValueError("E, sigma arrays must have the same length")
        h = C.c_void_p()
        _check(lib().hadros_sigma_from_arrays(E.ctypes.data, None if g is None else g.ctypes.data,
                                              s.ctypes.data, int(E.size), C.byref(h)))
        return cls(h.value)

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise HadrosError(abi.E_STATE, "sigma table was closed")
        return self._h

    def info(self) -> tuple[int, float, float]:
        n, lo, hi = C.c_int32(), C.c_double(), C.c_double()
        _check(lib().hadros_sigma_info(self.handle, C.byref(n), C.byref(lo), C.byref(hi)))
        return n.value, lo.value, hi.value

    def sigma_cm2(self, E: float) -> float:
        out = C.c_double()
        _check(lib().hadros_sigma_eval_cm2(self.handle, float(E), C.byref(out)))
        return out.value

    def close(self) -> None:
        if self._h:
            lib().hadros_sigma_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def n_bins_of(p: HadrosParams) -> int:
    return 1 if p.spectral_kind == 0 else max(int(p.n_bins), 1)


def spectral_bins(p: HadrosParams, sigma: SigmaTable) -> dict:
    """The bins integrate_kerr_ray_spectral uses: E_mid, dE, weight, valid."""
    B = n_bins_of(p)
    E, d, w = (np.zeros(B) for _ in range(3))
    v = np.zeros(B, dtype=np.int8)
    n = C.c_int32()
    _check(lib().hadros_spectral_bins(C.byref(p), sigma.handle, E.ctypes.data, d.ctypes.data,
                                      w.ctypes.data, v.ctypes.data, C.byref(n)))
    return {"E_mid": E[:n.value], "dE": d[:n.value], "weight": w[:n.value], "valid": v[:n.value]}


OUTPUTS = ("tau", "P_surv", "I_obs", "fate", "steps", "attempts", "tau_E", "I_E")
MEV_OUTPUTS = abi.MEV_OUTPUTS


def _with_mev(outputs, cams) -> tuple:
    """The default outputs gain the MeV channel's when a camera computes it."""
    if outputs is OUTPUTS and any(int(c.mev_channel) for c in cams):
        return OUTPUTS + MEV_OUTPUTS
    return tuple(outputs)


def pack_paths(points: np.ndarray, npoints: np.ndarray) -> np.ndarray:
    """[rows, cap, 7] path buffer -> points packed back to back (cut at cap)."""
    cap = points.shape[1]
    return np.concatenate([points[k, :min(int(n), cap)] for k, n in enumerate(npoints)] or
                          [np.zeros((0, 7))])


def write_kgeo(path, p: HadrosParams, npoints, points, pixel_ids=None, fate=None, append: bool = False) -> None:
    """KGEO geodesic cache file (the reference's compute_kerr_geodesics format);
    append=True adds the rays to an existing file (batched writing)."""
    n = np.ascontiguousarray(npoints, dtype=np.int32)
    pts = np.ascontiguousarray(points, dtype=np.float64)
    ids = None if pixel_ids is None else np.ascontiguousarray(pixel_ids, dtype=np.int32)
    fa = None if fate is None else np.ascontiguousarray(fate, dtype=np.int8)
    _check(lib().hadros_write_kgeo_rays(str(path).encode(), C.byref(p), int(n.size),
                                        None if ids is None else ids.ctypes.data,
                                        None if fa is None else fa.ctypes.data, n.ctypes.data,
                                        pts.ctypes.data if pts.size else None, 1 if append else 0))


def read_kgeo(path) -> dict:
    """Read a KGEO file: nx, ny, a, and per ray pixel id, captured, npoints,
    alpha, beta, plus the packed points [sum(npoints), 7]."""
    nx, ny, nr = C.c_int32(), C.c_int32(), C.c_int32()
    a, npts = C.c_double(), C.c_int64()
    _check(lib().hadros_kgeo_info(str(path).encode(), C.byref(nx), C.byref(ny), C.byref(a),
                                  C.byref(nr), C.byref(npts)))
    R = nr.value
    out = {"pixel_ids": np.zeros(R, np.int32), "captured": np.zeros(R, np.int8),
           "npoints": np.zeros(R, np.int32), "alpha": np.zeros(R), "beta": np.zeros(R),
           "points": np.zeros((npts.value, 7))}
    _check(lib().hadros_read_kgeo(str(path).encode(), *(out[k].ctypes.data for k in
                                  ("pixel_ids", "captured", "npoints", "alpha", "beta", "points"))))
    out.update(nx=nx.value, ny=ny.value, a_spin=a.value)
    return out


class Context:
    """A CUDA device context (hadros_ctx): one stream and its buffers."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().hadros_ctx_create(int(device), C.byref(h)))
        self._h = h
        self.device = device

    def close(self) -> None:
        if self._h:
            lib().hadros_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise HadrosError(abi.E_STATE, "context was closed")
        return self._h

    def stats(self) -> dict:
        s = HadrosStats()
        _check(lib().hadros_ctx_stats(self.handle, C.byref(s)))
        return {name: getattr(s, name) for name, _ in s._fields_}

    def set_transfer(self, mode) -> None:
        """Mixed-precision transfer placement: "auto", "in_loop" or "deferred"."""
        m = {"auto": abi.TRANSFER_AUTO, "in_loop": abi.TRANSFER_IN_LOOP,
             "deferred": abi.TRANSFER_DEFERRED}.get(mode, mode)
        _check(lib().hadros_ctx_set_transfer(self.handle, int(m)))

    def set_attempt_budget(self, attempts_per_ray: int) -> None:
        _check(lib().hadros_ctx_set_attempt_budget(self.handle, int(attempts_per_ray)))

    def image(self, p: HadrosParams, sigma: SigmaTable, pixel_ids=None,
              outputs=OUTPUTS) -> dict:
        """Trace an image (or a pixel list) into host numpy arrays; the default
        outputs gain tau_mev, P_surv_mev, I_obs_mev, r_nu and leakage when
        p.mev_channel is set."""
        outputs = _with_mev(outputs, [p])
        B = n_bins_of(p)
        P = int(p.nx) * int(p.ny) if pixel_ids is None else len(pixel_ids)
        fdt = np.float32 if p.precision == PRECISION_MIXED else np.float64
        shapes = {"tau": (P, np.float64), "P_surv": (P, np.float64), "I_obs": (P, np.float64),
                  "fate": (P, np.int8), "steps": (P, np.int32), "attempts": (P, np.int32),
                  "tau_E": ((P, B), fdt), "I_E": ((P, B), np.float64)}
        shapes.update({k: (P, np.float64) for k in MEV_OUTPUTS})
        res = {k: np.zeros(shapes[k][0], dtype=shapes[k][1]) for k in outputs}
        out = HadrosImageOut()
        for k, arr in res.items():
            setattr(out, k, arr.ctypes.data)
        if pixel_ids is None:
            _check(lib().hadros_image(self.handle, C.byref(p), sigma.handle, C.byref(out)))
        else:
            ids = np.ascontiguousarray(pixel_ids, dtype=np.int32)
            _check(lib().hadros_image_pixels(self.handle, C.byref(p), sigma.handle,
                                             ids.ctypes.data, int(ids.size), C.byref(out)))
        return res

    def batch(self, cams: list, sigma: SigmaTable, outputs=OUTPUTS) -> list[dict]:
        """Trace many cameras in one launch; returns one dict per camera."""
        outputs = _with_mev(outputs, cams)
        n = len(cams)
        arr = (HadrosParams * n)(*cams)
        Ps = [int(c.nx) * int(c.ny) for c in cams]
        Bs = [n_bins_of(c) for c in cams]
        P, PB = sum(Ps), sum(a * b for a, b in zip(Ps, Bs))
        fdt = np.float32 if cams[0].precision == PRECISION_MIXED else np.float64
        shapes = {"tau": (P, np.float64), "P_surv": (P, np.float64), "I_obs": (P, np.float64),
                  "fate": (P, np.int8), "steps": (P, np.int32), "attempts": (P, np.int32),
                  "tau_E": (PB, fdt), "I_E": (PB, np.float64)}
        shapes.update({k: (P, np.float64) for k in MEV_OUTPUTS})
        res = {k: np.zeros(shapes[k][0], dtype=shapes[k][1]) for k in outputs}
        out = HadrosImageOut()
        for k, a in res.items():
            setattr(out, k, a.ctypes.data)
        _check(lib().hadros_batch(self.handle, C.addressof(arr), n, sigma.handle, C.byref(out)))
        per, o, ob = [], 0, 0
        for Pc, Bc in zip(Ps, Bs):
            d = {}
            for k, a in res.items():
                d[k] = a[ob:ob + Pc * Bc].reshape(Pc, Bc) if k in ("tau_E", "I_E") else a[o:o + Pc]
            per.append(d)
            o += Pc
            ob += Pc * Bc
        return per

    def batch_pixels(self, cams: list, sigma: SigmaTable, pixel_lists: list, outputs=OUTPUTS) -> list[dict]:
        """Pixel subsets of many cameras in one launch (hadros_batch_pixels):
        camera c traces pixel_lists[c]; returns one dict per camera, rows in
        list order."""
        outputs = _with_mev(outputs, cams)
        n = len(cams)
        if len(pixel_lists) != n:
            raise ValueError("one pixel list per camera")
        arr = (HadrosParams * n)(*cams)
        lists = [np.ascontiguousarray(ids, dtype=np.int32) for ids in pixel_lists]
        counts = np.array([ids.size for ids in lists], dtype=np.int32)
        ids = np.concatenate(lists) if lists else np.zeros(0, np.int32)
        Bs = [n_bins_of(c) for c in cams]
        P, PB = int(counts.sum()), int(sum(int(c) * b for c, b in zip(counts, Bs)))
        fdt = np.float32 if cams[0].precision == PRECISION_MIXED else np.float64
        shapes = {"tau": (P, np.float64), "P_surv": (P, np.float64), "I_obs": (P, np.float64),
                  "fate": (P, np.int8), "steps": (P, np.int32), "attempts": (P, np.int32),
                  "tau_E": (PB, fdt), "I_E": (PB, np.float64)}
        shapes.update({k: (P, np.float64) for k in MEV_OUTPUTS})
        res = {k: np.zeros(shapes[k][0], dtype=shapes[k][1]) for k in outputs}
        out = HadrosImageOut()
        for k, a in res.items():
            setattr(out, k, a.ctypes.data)
        _check(lib().hadros_batch_pixels(self.handle, C.addressof(arr), n, sigma.handle, ids.ctypes.data,
                                         counts.ctypes.data, C.byref(out)))
        per, o, ob = [], 0, 0
        for Pc, Bc in zip(counts, Bs):
            Pc = int(Pc)
            d = {}
            for k, a in res.items():
                d[k] = a[ob:ob + Pc * Bc].reshape(Pc, Bc) if k in ("tau_E", "I_E") else a[o:o + Pc]
            per.append(d)
            o += Pc
            ob += Pc * Bc
        return per

    def trace_paths(self, p: HadrosParams, pixel_ids=None, max_points: int = 50000) -> dict:
        """Record every pixel's path points (r, theta, x, y, z, dl, redshift).

        Returns ``points`` [rows, max_points, 7], ``npoints`` and ``fate``."""
        rows = int(p.nx) * int(p.ny) if pixel_ids is None else len(pixel_ids)
        pts = np.zeros((rows, max_points, 7))
        n = np.zeros(rows, dtype=np.int32)
        f = np.zeros(rows, dtype=np.int8)
        ids = None if pixel_ids is None else np.ascontiguousarray(pixel_ids, dtype=np.int32)
        _check(lib().hadros_trace_paths(self.handle, C.byref(p), None if ids is None else ids.ctypes.data,
                                        0 if ids is None else int(ids.size), int(max_points),
                                        pts.ctypes.data, n.ctypes.data, f.ctypes.data))
        return {"points": pts, "npoints": n, "fate": f}

    def transfer_paths(self, p: HadrosParams, sigma: SigmaTable, npoints, points, fate=None,
                       outputs=("tau", "P_surv", "I_obs", "fate", "steps", "tau_E", "I_E")) -> dict:
        """Transfer over cached paths: points packed back to back [sum(npoints), 7]
        (with the MeV channel's outputs when p computes it)."""
        if int(p.mev_channel):
            outputs = tuple(outputs) + tuple(k for k in MEV_OUTPUTS if k not in outputs)
        n = np.ascontiguousarray(npoints, dtype=np.int32)
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 7)
        if pts.shape[0] != int(n.sum()):
            raise ValueError("points must hold sum(npoints) rows of 7 doubles")
        fa = None if fate is None else np.ascontiguousarray(fate, dtype=np.int8)
        P, B = int(n.size), n_bins_of(p)
        fdt = np.float32 if p.precision == PRECISION_MIXED else np.float64
        shapes = {"tau": (P, np.float64), "P_surv": (P, np.float64), "I_obs": (P, np.float64),
                  "fate": (P, np.int8), "steps": (P, np.int32),
                  "tau_E": ((P, B), fdt), "I_E": ((P, B), np.float64)}
        shapes.update({k: (P, np.float64) for k in MEV_OUTPUTS})
        res = {k: np.zeros(shapes[k][0], dtype=shapes[k][1]) for k in outputs}
        out = HadrosImageOut()
        for k, a in res.items():
            setattr(out, k, a.ctypes.data)
        _check(lib().hadros_transfer_paths(self.handle, C.byref(p), sigma.handle, P, n.ctypes.data,
                                           None if fa is None else fa.ctypes.data,
                                           pts.ctypes.data if pts.size else None, C.byref(out)))
        return res

    def plan(self, cams: list, sigma: SigmaTable, schedule=None) -> "Plan":
        """Upload a scan once (see hadros_plan_create)."""
        return Plan(self, cams, sigma, schedule)

    def image_device(self, p: HadrosParams, sigma: SigmaTable, out: dict, stream=None) -> None:
        """Enqueue an image into device buffers (torch tensors or raw pointers)."""
        o = HadrosImageOut()
        for k, v in out.items():
            setattr(o, k, v if isinstance(v, int) else v.data_ptr())
        _check(lib().hadros_image_device(self.handle, C.byref(p), sigma.handle, C.byref(o), _ptr_stream(stream)))

    def pixels_device(self, p: HadrosParams, sigma: SigmaTable, ids, out: dict, n: int | None = None,
                      stream=None) -> None:
        """Enqueue the exact trace of a DEVICE pixel-id list (int32 tensor or
        pointer; first n ids, default all) into device buffers in list order."""
        o = HadrosImageOut()
        for k, v in out.items():
            setattr(o, k, v if isinstance(v, int) else v.data_ptr())
        count = int(ids.numel()) if n is None else int(n)
        ptr = ids if isinstance(ids, int) else ids.data_ptr()
        _check(lib().hadros_image_pixels_device(self.handle, C.byref(p), sigma.handle, C.c_void_p(ptr), count,
                                                C.byref(o), _ptr_stream(stream)))

    def synchronize(self) -> None:
        _check(lib().hadros_ctx_synchronize(self.handle))


def schedule(**kw) -> HadrosSchedule:
    """hadros_schedule_default() with overrides (blocks_per_sm, order, ...)."""
    sc = HadrosSchedule()
    lib().hadros_schedule_default(C.byref(sc))
    for k, v in kw.items():
        setattr(sc, k, int(v))
    return sc


# cudaStreamLegacy: the legacy default stream, named explicitly because a
# NULL stream at the image entry points means the context's own stream.
_STREAM_LEGACY = 1


def _ptr_stream(stream):
    """The cudaStream_t to pass for `stream` (a torch stream or a raw handle;
    None = the context's stream).  Torch's default stream has handle 0, which
    the image entry points would read as the context's own non-blocking
    stream, unordered with the caller's work; it goes as cudaStreamLegacy."""
    if stream is None:
        return None
    h = stream if isinstance(stream, int) else stream.cuda_stream
    return C.c_void_p(h if h else _STREAM_LEGACY)


class Plan:
    """A scan uploaded once; launch() only enqueues the kernel (capturable)."""

    def __init__(self, ctx: Context, cams: list, sigma: SigmaTable, sched=None):
        self.cams = list(cams)
        arr = (HadrosParams * len(self.cams))(*self.cams)
        h = C.c_void_p()
        _check(lib().hadros_plan_create(ctx.handle, C.addressof(arr), len(self.cams), sigma.handle,
                                        None if sched is None else C.byref(sched), C.byref(h)))
        self._h = h
        self.ctx = ctx
        n, nb, g, b = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int32()
        _check(lib().hadros_plan_info(h, C.byref(n), C.byref(nb), C.byref(g), C.byref(b)))
        self.n_pixels, self.n_pixel_bins, self.grid, self.blocks_per_sm = n.value, nb.value, g.value, b.value

    def alloc(self, torch, device=None, outputs=OUTPUTS) -> dict:
        """Device output tensors for this plan."""
        P, PB = self.n_pixels, self.n_pixel_bins
        f32 = self.cams[0].precision == PRECISION_MIXED
        spec = {"tau": (P, torch.float64), "P_surv": (P, torch.float64), "I_obs": (P, torch.float64),
                "fate": (P, torch.int8), "steps": (P, torch.int32), "attempts": (P, torch.int32),
                "tau_E": (PB, torch.float32 if f32 else torch.float64), "I_E": (PB, torch.float64)}
        spec.update({k: (P, torch.float64) for k in MEV_OUTPUTS})
        outputs = _with_mev(outputs, self.cams)
        return {k: torch.empty(spec[k][0], dtype=spec[k][1], device=device) for k in outputs}

    def launch(self, out: dict, stream=None) -> None:
        o = HadrosImageOut()
        for k, v in out.items():
            setattr(o, k, v if isinstance(v, int) else v.data_ptr())
        _check(lib().hadros_plan_launch(self._h, C.byref(o), _ptr_stream(stream)))

    def counters(self, stream=None) -> dict:
        st, at, ab = C.c_int64(), C.c_int64(), C.c_int32()
        _check(lib().hadros_plan_counters(self._h, _ptr_stream(stream), C.byref(st), C.byref(at),
                                          C.byref(ab)))
        return {"accepted_steps": st.value, "attempts": at.value, "aborted": ab.value}

    def close(self) -> None:
        if self._h:
            lib().hadros_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
