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


def _noalloc(hb, torch, p, sigma, mev: bool = False, calls: int = 1) -> tuple[dict, list[int]]:
    """`calls` no-alloc calls into the same pre-filled buffers; returns the
    last call's outputs and the device's free bytes around each call."""
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
    if mev:
        bufs.update({k: torch.full((P,), -7.0, dtype=torch.float64, device=dev) for k in hb.MEV_OUTPUTS})
    out = hb.HadrosImageOut()
    for k, t in bufs.items():
        setattr(out, k, t.data_ptr())
    free = []
    for _ in range(calls):
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info(0)[0])
        rc = hb.lib().hadros_image_device_noalloc(C.byref(p), sigma.handle, C.byref(out),
                                                   C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0, hb.lib().hadros_last_error().decode()
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info(0)[0])
    return {k: t.cpu().numpy() for k, t in bufs.items()}, free


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
            got, _ = _noalloc(hb, torch, p, sigma_table)
            assert_parity(got, ref, rtol, f"noalloc {precision} call {call}",
                          p_absolute=(precision == "mixed"))
            np.testing.assert_array_equal(got["attempts"], ref["attempts"])


def test_noalloc_allocates_nothing_and_runs_the_mev_channel(hb, gpu_ctx, sigma_table):
    """A warm call leaves the device's free memory unchanged, and the MeV
    channel's outputs equal the ordinary entry point's."""
    import torch
    from hadros_b200 import workloads as W
    torch.cuda.set_device(0)
    p = hb.params(**W.mixed_512(nx=6, ny=5, h=0.05, precision="mixed", fast=False, mev_channel=1))
    ref = gpu_ctx.image(p, sigma_table)
    got, free = _noalloc(hb, torch, p, sigma_table, mev=True, calls=3)
    # the first call may load the library's kernels; the later ones allocate nothing
    assert free[2] == free[3] and free[4] == free[5], f"free device bytes changed: {free}"
    errs = assert_parity(got, ref, RTOL_MIXED, "noalloc mev", p_absolute=True)
    assert all(k in errs for k in hb.MEV_OUTPUTS)


def test_noalloc_at_its_limits(hb, gpu_ctx):
    """64 bins with a 1024-row sigma table in mixed precision: the largest
    request the entry point accepts (the bins' accumulators then fill most of
    the block's shared memory), twice in a row."""
    import torch
    from hadros_b200 import workloads as W
    torch.cuda.set_device(0)
    E = np.logspace(4.0, 12.0, 1024)
    s = 7.84e-36 * E ** 0.363
    big = hb.SigmaTable.from_arrays(E, s, s / 0.389379e-27)
    p = hb.params(**W.production_point(nx=4, ny=3, h=0.05, n_bins=64, fast=False))
    ref = gpu_ctx.image(p, big)
    for call in range(2):
        got, _ = _noalloc(hb, torch, p, big)
        assert_parity(got, ref, RTOL_MIXED, f"noalloc limits call {call}", p_absolute=True)


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
