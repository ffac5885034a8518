"""Surrogate network on the GPU: the training kernels against the CPU oracle
(forward outputs and gradients), a training run that learns, the sample
features against their definition, and the tcgen05 inference kernel against
the training forward pass (per sample and per pixel)."""
from __future__ import annotations

import ctypes as C
import math
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent.parent / "oracle"))
import mlp_oracle as M  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    torch.cuda.set_device(0)
    return torch


def _vp(t):
    return C.c_void_p(t.data_ptr())


def _random_master(seed, bias_scale=0.2):
    from hadros_b200 import surrogate as S
    rng = np.random.default_rng(seed)
    m = S.init_master(seed)
    for name in ("b1", "b2", "b3", "b4", "b5", "Ws"):
        o, n = M.OFF[name]
        m[o:o + n] = rng.uniform(-bias_scale, bias_scale, n)
    o, n = M.OFF["W5"]
    m[o:o + n] *= 10.0
    return m.astype(np.float32)


def _features(torch, hb, n, seed):
    rng = np.random.default_rng(seed)
    raw = rng.normal(size=(n, 16)).astype(np.float32)
    raw[:, 5:13] = 0.0
    raw[np.arange(n), 5 + rng.integers(0, 8, n)] = 1.0
    norm = hb.abi.HadrosMlpNorm()
    for j in range(16):
        norm.feat_inv_sd[j] = 1.0
    raw_t = torch.from_numpy(raw).cuda()
    X = torch.empty((n, 64), dtype=torch.bfloat16, device="cuda")
    assert hb.lib().hadros_mlp_featurize(_vp(raw_t), n, C.byref(norm), _vp(X), None) == 0
    return raw, X


def _forward(torch, hb, master_np, X):
    L = hb.lib()
    n = X.shape[0]
    master = torch.from_numpy(master_np).cuda()
    packed = torch.empty(int(L.hadros_mlp_packed_count()), dtype=torch.bfloat16, device="cuda")
    assert L.hadros_mlp_pack(_vp(master), _vp(packed), None) == 0
    ws = torch.empty(int(L.hadros_mlp_workspace_bytes(n)), dtype=torch.uint8, device="cuda")
    out = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    assert L.hadros_mlp_forward(_vp(master), _vp(packed), _vp(X), n, _vp(ws), _vp(out), None) == 0
    return master, packed, ws, out


def test_featurize_matches_oracle_split(hb, torch):
    raw, X = _features(torch, hb, 777, 1)
    ref = M.split_features(raw, np.zeros(16), np.ones(16))
    got = X.float().cpu().numpy().astype(np.float64)
    np.testing.assert_array_equal(got[:, :32], ref[:, :32])
    # Fourier columns: the GPU's sin/cos may round to the neighbouring BF16 value
    assert np.abs(got[:, 32:] - ref[:, 32:]).max() <= 2.0 ** -8
    assert np.mean(got[:, 32:] != ref[:, 32:]) < 0.02


@pytest.mark.parametrize("n", [200, 1024, 4100])
def test_forward_matches_oracle(hb, torch, n):
    master_np = _random_master(5)
    raw, X = _features(torch, hb, n, 2)
    _, _, _, out = _forward(torch, hb, master_np, X)
    torch.cuda.synchronize()
    got = out.cpu().numpy().astype(np.float64)
    ref, _ = M.forward(master_np, X.float().cpu().numpy())
    # SiLU runs in BF16 on the GPU with the hardware tanh approximation: some
    # activations land one BF16 step (2^-8 relative) from the oracle's, which
    # after four layers is ~0.5% of the output scale
    rel = np.sqrt(np.mean((got - ref) ** 2)) / np.sqrt(np.mean(ref ** 2))
    assert rel < 1e-2, rel
    assert np.abs(got - ref).max() < 0.05 * np.abs(ref).max()


def test_backward_matches_oracle(hb, torch):
    """The GPU gradient of sum(dout * out) against the oracle's, per block of
    the master layout (BF16 rounding points emulated by the oracle)."""
    n = 2048
    master_np = _random_master(7)
    raw, X = _features(torch, hb, n, 3)
    master, packed, ws, out = _forward(torch, hb, master_np, X)
    rng = np.random.default_rng(4)
    dout_np = rng.normal(size=(n, 2)).astype(np.float32) / n
    dout = torch.from_numpy(dout_np).cuda()
    grad = torch.zeros(int(hb.lib().hadros_mlp_param_count()), dtype=torch.float32, device="cuda")
    assert hb.lib().hadros_mlp_backward(_vp(packed), _vp(X), n, _vp(dout), _vp(ws), _vp(grad), None) == 0
    torch.cuda.synchronize()
    g = grad.cpu().numpy().astype(np.float64)
    _, cache = M.forward(master_np, X.float().cpu().numpy())
    gr = M.pack_grad(M.backward(cache, dout_np.astype(np.float64)))
    for name, (o, k) in M.OFF.items():
        a, b = g[o:o + k], gr[o:o + k]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        cos = float(a @ b) / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30)
        assert rel < 5e-2 and cos > 0.998, (name, rel, cos)
    assert not np.any(g[M.PARAMS_USED:])


def test_training_learns_a_smooth_function(hb, torch):
    """Adam through hadros_mlp_train_step fits a smooth 2-output function of the
    features: the loss falls by more than 30x."""
    from hadros_b200 import surrogate as S
    n = 32768
    rng = np.random.default_rng(8)
    raw = rng.uniform(-1, 1, size=(n, 16)).astype(np.float32)
    raw[:, 5:13] = 0.0
    raw[np.arange(n), 5 + rng.integers(0, 8, n)] = 1.0
    y = np.stack([np.sin(2 * raw[:, 0]) + 0.5 * raw[:, 1] ** 2 + 0.3 * raw[:, 15],
                  raw[:, 0] * raw[:, 1] - 0.7 * raw[:, 4] + 0.2 * raw[:, 5]], axis=1).astype(np.float32)
    sur = S.Surrogate(members=1, seed=3)
    hist = sur.fit(torch.from_numpy(raw).cuda(), torch.from_numpy(y).cuda(), epochs=12, batch=4096, lr=3e-3)
    h = hist[0]
    assert all(math.isfinite(v) for v in h)
    assert h[-1] < h[0] / 30.0, h


def test_raw_features_match_definition(hb, torch, sigma_table):
    from hadros_b200 import surrogate as S
    p = hb.params(nx=37, ny=23, fov_deg=25.0, r_obs_rg=60.0, a_spin=0.7, theta_obs_deg=35.0,
                  rho0_gcm3=3e10, r0_rg=12.0, H_over_R=0.4, profile="powerlaw_funnel",
                  spectral="powerlaw_cutoff", n_bins=8)
    ids = np.array([0, 5, 36, 37, 400, 850], dtype=np.int32)
    raw = S.raw_features(p, sigma_table, ids).cpu().numpy()
    bins = hb.spectral_bins(p, sigma_table)
    B = 8
    tan = math.tan(0.5 * 25.0 * math.pi / 180.0) * 60.0
    for k, pid in enumerate(ids):
        i, j = pid % 37, pid // 37
        for b in range(B):
            f = raw[k * B + b]
            np.testing.assert_allclose(f[0], ((2 * i + 1) / 37 - 1.0) * tan, rtol=1e-5, atol=1e-5)
            np.testing.assert_allclose(f[1], ((2 * j + 1) / 23 - 1.0) * tan, rtol=1e-5, atol=1e-5)
            np.testing.assert_allclose(f[2:5], [0.7, math.cos(35 * math.pi / 180), math.log10(3e10)], rtol=1e-6)
            onehot = np.zeros(8)
            onehot[3] = 1.0
            np.testing.assert_array_equal(f[5:13], onehot)
            np.testing.assert_allclose(f[13:16], [12.0, 0.4, math.log10(bins["E_mid"][b])], rtol=1e-6)


def _random_surrogate(hb, torch, members, seed):
    from hadros_b200 import surrogate as S
    sur = S.Surrogate(members=members, seed=seed)
    for k, net in enumerate(sur.nets):
        net.load_master(_random_master(seed * 10 + k, bias_scale=0.1))
    nm = hb.abi.HadrosMlpNorm()
    mu = [0.0, 0.0, 0.9, 0.5, 10.5] + [0.0] * 8 + [10.0, 0.3, 8.0]
    sd = [10.0, 10.0, 0.1, 0.3, 1.0] + [1.0] * 8 + [3.0, 0.1, 2.0]
    for j in range(16):
        nm.feat_mu[j] = mu[j]
        nm.feat_inv_sd[j] = 1.0 / sd[j]
    nm.out_mu[0], nm.out_sd[0] = 2.0, 3.0
    nm.out_mu[1], nm.out_sd[1] = -60.0, 4.0
    nm.out_floor[0], nm.out_floor[1] = 1e-6, 0.0
    sur.norm = nm
    return sur


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("members,n_bins,nx,ny,begin,end,spread_of", [
    (1, 8, 24, 24, 0, None, 0),
    (2, 16, 33, 17, 0, None, 0),
    (3, 64, 20, 20, 37, 333, 0),
    (4, 1, 50, 30, 0, None, 0),
    (3, 32, 16, 16, 0, None, 1),
])
def test_umma_inference_matches_training_forward(hb, torch, sigma_table, members, n_bins, nx, ny, begin, end,
                                                 spread_of, schedule):
    """The fused tcgen05 kernel and the mma.sync training forward pass compute
    the same network: per-sample ensemble means within BF16 rounding, and the
    per-pixel aggregates and spread as the host forms them from the forward
    pass's per-member outputs."""
    from hadros_b200 import surrogate as S
    sur = _random_surrogate(hb, torch, members, seed=members)
    kw = dict(nx=nx, ny=ny, profile="collapsar_ndaf_like", a_spin=0.95, theta_obs_deg=40.0, rho0_gcm3=1e11)
    if n_bins == 1:
        kw.update(spectral="monochromatic")
    else:
        kw.update(spectral="powerlaw_cutoff", n_bins=n_bins)
    p = hb.params(**kw)
    P = nx * ny
    end = P if end is None else end
    old = hb.lib().hadros_surrogate_schedule(-1)
    assert hb.lib().hadros_surrogate_schedule(schedule) == 0
    try:
        res = sur.image(p, sigma_table, pixel_begin=begin, pixel_end=end, threshold=0.05, spread_of=spread_of)
        torch.cuda.synchronize()
    finally:
        hb.lib().hadros_surrogate_schedule(old)
    torch.cuda.synchronize()
    cnt = res["counters"].cpu().numpy()
    assert cnt[1] == 0, "inference kernel aborted"
    ids = np.arange(begin, end, dtype=np.int32)
    raw = S.raw_features(p, sigma_table, ids)
    fw = sur.forward(raw).cpu().numpy().astype(np.float64)      # [K][n*B][2]
    B = n_bins
    mean = fw.mean(0)
    got_t = res["ln_tau_E"].cpu().numpy().reshape(-1)
    got_i = res["ln_I_E"].cpu().numpy().reshape(-1)
    for got, ref, scale in ((got_t, mean[:, 0], 3.0), (got_i, mean[:, 1], 4.0)):
        err = np.abs(got - ref)
        assert np.sqrt(np.mean(err ** 2)) < 0.02 * scale, np.sqrt(np.mean(err ** 2))
        assert err.max() < 0.2 * scale, err.max()
    bins = hb.spectral_bins(p, sigma_table)
    valid = (bins["valid"] != 0) & (bins["dE"] > 0)
    lnde = np.where(valid, np.log(np.where(valid, bins["dE"], 1.0)), -np.inf)
    if spread_of == 0:
        L_k = np.log(np.sum(np.exp(fw[:, :, 1].reshape(members, -1, B) + lnde), axis=2))   # [K][n]
    else:
        wv = np.where(valid, bins["weight"], 0.0)
        L_k = np.log(np.sum(np.exp(fw[:, :, 0].reshape(members, -1, B)) * wv, axis=2) / wv.sum())
    spread_ref = L_k.std(0)
    spread = res["spread"].cpu().numpy()
    if members == 1:
        assert not np.any(spread)
    assert np.abs(spread - spread_ref).max() < 0.05 + 0.05 * spread_ref.max()
    I_ref = np.exp(np.log(np.sum(np.exp(got_i.reshape(-1, B) + lnde), axis=1)))
    np.testing.assert_allclose(res["I_obs"].cpu().numpy(), I_ref, rtol=1e-4)
    w = np.where(valid, bins["weight"], 0.0)
    tau_E = np.maximum(np.exp(got_t.reshape(-1, B)) - 1e-6, 0.0)
    np.testing.assert_allclose(res["tau"].cpu().numpy(), (tau_E * w).sum(1) / w.sum(), rtol=1e-4)
    np.testing.assert_allclose(res["P_surv"].cpu().numpy(), (np.exp(-tau_E) * w).sum(1) / w.sum(),
                               rtol=1e-4, atol=1e-12)
    fb = np.sort(res["fallback_ids"][:int(cnt[0])].cpu().numpy())
    expect = ids[spread > 0.05]       # the kernel's own spread decides
    np.testing.assert_array_equal(fb, expect)


@pytest.mark.parametrize("members,n_bins", [(2, 8), (4, 64)])
def test_umma_inference_matches_oracle(hb, torch, sigma_table, members, n_bins):
    """The fused tcgen05 inference kernel against the CPU oracle's forward
    pass (oracle/mlp_oracle.py with the BF16 rounding points of the kernels)
    on the kernel's own input rows: per sample, the ensemble means of ln tau_E
    and ln I_E differ by FP32 summation order and the hardware tanh only (an
    activation that lands near a BF16 rounding boundary can round to the
    neighbouring BF16 value, a 2^-8 relative step).  The per-pixel spread of
    ln I_obs is the members' standard deviation of a log-sum-exp over bins;
    both maps are 1-Lipschitz in the largest per-member difference, so the
    spread may differ by at most the per-output bound, in ln I units."""
    from hadros_b200 import surrogate as S
    sur = _random_surrogate(hb, torch, members, seed=20 + members)
    nx, ny = 20, 16
    p = hb.params(nx=nx, ny=ny, profile="collapsar_ndaf_like", a_spin=0.95, theta_obs_deg=40.0, rho0_gcm3=1e11,
                  spectral="powerlaw_cutoff", n_bins=n_bins)
    res = sur.image(p, sigma_table, threshold=1e30)
    torch.cuda.synchronize()
    assert res["counters"].cpu().numpy()[1] == 0, "inference kernel aborted"
    P, B = nx * ny, n_bins
    raw = S.raw_features(p, sigma_table, np.arange(P, dtype=np.int32))
    X = sur.featurize(raw).float().cpu().numpy().astype(np.float64)
    nm = sur.norm
    mu = np.array([nm.out_mu[0], nm.out_mu[1]])
    sd = np.array([nm.out_sd[0], nm.out_sd[1]])
    ys = np.stack([M.forward(net.master.cpu().numpy(), X)[0] * sd + mu for net in sur.nets])   # [K][n][2]
    mean = ys.mean(0)
    got = np.stack([res["ln_tau_E"].cpu().numpy().reshape(-1), res["ln_I_E"].cpu().numpy().reshape(-1)], axis=1)
    err = np.abs(got - mean) / sd                       # in units of the outputs' spread
    rms, worst = np.sqrt(np.mean(err ** 2, axis=0)), err.max(axis=0)
    bins = hb.spectral_bins(p, sigma_table)
    valid = (bins["valid"] != 0) & (bins["dE"] > 0)
    lnde = np.where(valid, np.log(np.where(valid, bins["dE"], 1.0)), -np.inf)
    L_k = np.log(np.sum(np.exp(ys[:, :, 1].reshape(members, P, B) + lnde), axis=2))   # [K][P]
    spread_ref = L_k.std(0)
    d_spread = np.abs(res["spread"].cpu().numpy() - spread_ref) / sd[1]    # in ln I_E sd units
    stats = (f"rms {rms.tolist()} max {worst.tolist()} (output sd units); spread |diff| rms "
             f"{np.sqrt(np.mean(d_spread ** 2)):.3e} max {d_spread.max():.3e} (ln I_E sd units; spread up to "
             f"{spread_ref.max() / sd[1]:.3e})")
    print(stats)
    # a BF16 step is 2^-8 = 0.4% of a unit-scale value: a few steps at worst
    assert rms.max() < 5e-3 and worst.max() < 2e-2, stats
    assert np.sqrt(np.mean(d_spread ** 2)) < 5e-3 and d_spread.max() < 2e-2, stats
