"""hadros_image_device_noalloc: the entry point for callers that cannot call
cudaMalloc (their device memory belongs to another allocator or to a fixed
budget).  It keeps its scratch in a static device array inside the library,
so the caller passes only parameters, the sigma table and output buffers.

Checked through the C ABI against the ordinary entry point (hadros_image),
with the tolerances of the other parity tests, on two calls in a row (the
shared scratch keeps the previous call's contents, so the second call shows
that every call starts clean).  This file is collected last."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from parity import RTOL_FP64, RTOL_MIXED, assert_parity

pytestmark = pytest.mark.gpu


def _noalloc(hb, torch, p, sigma) -> dict:
    P, B = p.nx * p.ny, hb.n_bins_of(p)
    dev = torch.device("cuda", 0)
    fdt = torch.float32 if p.precision == hb.PRECISION_MIXED else torch.float64
    bufs = {"tau": torch.full((P,), -7.0, dtype=torch.float64, device=dev),
            "P_surv": torch.full((P,), -7.0, dtype=torch.float64, device=dev),
            "I_obs": torch.full((P,), -7.0, dtype=torch.float64, device=dev),
            "fate": torch.full((P,), -1, dtype=torch.int8, device=dev),
            "steps": torch.full((P,), -1, dtype=torch.int32, device=dev),
            "attempts": torch.full((P,), -1, dtype=torch.int32, device=dev),
            "tau_E": torch.full((P, B), -7.0, dtype=fdt, device=dev),
            "I_E": torch.full((P, B), -7.0, dtype=torch.float64, device=dev)}
    out = hb.HadrosImageOut()
    for k, t in bufs.items():
        setattr(out, k, t.data_ptr())
    torch.cuda.synchronize()
    rc = hb.lib().hadros_image_device_noalloc(C.byref(p), sigma.handle, C.byref(out),
                                               C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, hb.lib().hadros_last_error().decode()
    torch.cuda.synchronize()
    return {k: t.cpu().numpy() for k, t in bufs.items()}


@pytest.mark.parametrize("precision,rtol", [("fp64", RTOL_FP64), ("mixed", RTOL_MIXED)])
def test_noalloc_matches_ordinary_entry_point_twice(hb, gpu_ctx, sigma_table, precision, rtol):
    import torch
    from hadros_b200 import workloads as W
    torch.cuda.set_device(0)
    # the no-alloc entry point runs the reference-arithmetic kernel (fast=False)
    cases = [W.mixed_512(nx=9, ny=7, h=0.05, precision=precision, fast=False),
             W.plain_tracer_32(nx=5, ny=6, r_obs_rg=60.0, r_max_rg=120.0, fov_deg=25.0, h=0.05,
                               precision=precision, fast=False)]
    for kw in cases:
        p = hb.params(**kw)
        ref = gpu_ctx.image(p, sigma_table)
        for call in range(2):
            got = _noalloc(hb, torch, p, sigma_table)
            assert_parity(got, ref, rtol, f"noalloc {precision} call {call}",
                          p_absolute=(precision == "mixed"))
            np.testing.assert_array_equal(got["attempts"], ref["attempts"])


def test_noalloc_rejects_sizes_beyond_its_limits(hb, sigma_table):
    import torch
    torch.cuda.set_device(0)
    out = hb.HadrosImageOut()
    p = hb.params(spectral="powerlaw_cutoff", n_bins=65, nx=2, ny=2, fast=False)
    rc = hb.lib().hadros_image_device_noalloc(C.byref(p), sigma_table.handle, C.byref(out), None)
    assert rc == 1 and b"64 spectral bins" in hb.lib().hadros_last_error()
    E = np.logspace(4, 12, 1025)
    big = hb.SigmaTable.from_arrays(E, 1e-35 * E ** 0.3)
    rc = hb.lib().hadros_image_device_noalloc(C.byref(hb.params(nx=2, ny=2, fast=False)), big.handle,
                                               C.byref(out), None)
    assert rc == 1 and b"1024" in hb.lib().hadros_last_error()
