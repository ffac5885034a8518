"""Learned surrogate of the tracer for parameter scans (no counterpart in the
reference).

An ensemble of small BF16 tensor-core MLPs (include/hadros_b200.h,
"surrogate network") predicts ln tau_E and ln I_E of each (pixel, bin) from
the camera, medium and energy; the pixels whose ensemble spread of ln I_obs
exceeds a threshold are traced exactly, and the exact tracer also judges a
random subset of every image.  PyTorch only holds device memory and streams
here: every forward, backward, optimizer and inference step is a call into
libhadros_b200.so.

    sur = Surrogate(members=4)
    raw, y = trace_samples(ctx, sigma, train_cams, pixels_per_cam=512)
    sur.fit(raw, y, epochs=20)
    res = sur.image(p, sigma)                  # device tensors + fallback ids
    img = sur.image_with_fallback(ctx, p, sigma)
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import HadrosError, _check, abi, lib, n_bins_of
from .abi import HadrosAdam, HadrosMlpNorm, HadrosSurrogateOut

N_FEATURES = 16
N_INPUT = 64                      # BF16 input columns: hi, lo, Fourier features
N_OUT = 2
PROFILE_FEATURES = range(5, 13)   # one-hot torus profile kind
TAU_FLOOR = 1.0e-6                # ln(tau_E + floor): tau below it is transparent
I_FLOOR_REL = 1.0e-12             # ln(I_E + floor), floor relative to the largest I_E


def _torch():
    import torch
    return torch


def _vp(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def _stream_ptr(stream) -> C.c_void_p:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def init_master(seed: int) -> np.ndarray:
    """FP32 master parameters of one network: uniform fan-in weights, zero
    biases and skip, a small last layer."""
    L = lib()
    n = int(L.hadros_mlp_param_count())
    off = layout()
    rng = np.random.default_rng(seed)
    m = np.zeros(n, dtype=np.float32)
    for name, fan_in in (("W1", N_INPUT), ("W2", 256), ("W3", 256), ("W4", 256), ("W5", 256)):
        a, b = off[name]
        lim = math.sqrt(6.0 / fan_in) * (0.1 if name == "W5" else 1.0)
        m[a:b] = rng.uniform(-lim, lim, b - a)
    return m


def layout() -> dict:
    """Master-array slices {name: (begin, end)} of W1, b1, ..., Ws."""
    o = (C.c_int64 * 12)()
    _check(lib().hadros_mlp_layout(o, 12))
    names = ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4", "W5", "b5", "Ws")
    return {nm: (int(o[i]), int(o[i + 1])) for i, nm in enumerate(names)}


def make_norm(raw, targets, floors=(TAU_FLOOR, 0.0)) -> HadrosMlpNorm:
    """Feature and target standardization from a training set (torch tensors
    [n][16], [n][2] of ln values); one-hot and constant features are left as
    is.  `floors` are the constants added before the logarithm of each target."""
    torch = _torch()
    nm = HadrosMlpNorm()
    mu = raw.double().mean(0).cpu().numpy()
    sd = raw.double().std(0).cpu().numpy()
    for j in range(N_FEATURES):
        if j in PROFILE_FEATURES or sd[j] < 1e-12:
            nm.feat_mu[j] = 0.0 if j in PROFILE_FEATURES else float(mu[j])
            nm.feat_inv_sd[j] = 1.0
        else:
            nm.feat_mu[j] = float(mu[j])
            nm.feat_inv_sd[j] = float(1.0 / sd[j])
    tmu = targets.double().mean(0).cpu().numpy()
    tsd = targets.double().std(0).cpu().numpy()
    for o in range(N_OUT):
        nm.out_mu[o] = float(tmu[o])
        nm.out_sd[o] = float(max(tsd[o], 1e-6))
        nm.out_floor[o] = float(floors[o])
    del torch
    return nm


class Network:
    """One network's device state: FP32 master, BF16 working copy, Adam moments
    and gradient (views into the ensemble's stacked arrays when given)."""

    def __init__(self, device, seed: int, views: dict | None = None):
        torch = _torch()
        L = lib()
        self.device = torch.device(device)
        self.n_params = int(L.hadros_mlp_param_count())
        if views is None:
            views = {"master": torch.empty(self.n_params, dtype=torch.float32, device=self.device),
                     "packed": torch.empty(int(L.hadros_mlp_packed_count()), dtype=torch.bfloat16,
                                           device=self.device),
                     "m": torch.empty(self.n_params, dtype=torch.float32, device=self.device),
                     "v": torch.empty(self.n_params, dtype=torch.float32, device=self.device),
                     "grad": torch.empty(self.n_params, dtype=torch.float32, device=self.device)}
        self.master, self.packed = views["master"], views["packed"]
        self.m, self.v, self.grad = views["m"], views["v"], views["grad"]
        self.master.copy_(torch.from_numpy(init_master(seed)))
        self.m.zero_()
        self.v.zero_()
        self.grad.zero_()
        self.step = 0
        self.pack()

    def pack(self, stream=None) -> None:
        _check(lib().hadros_mlp_pack(_vp(self.master), _vp(self.packed), _stream_ptr(stream)))

    def load_master(self, master) -> None:
        torch = _torch()
        self.master.copy_(torch.as_tensor(np.asarray(master, dtype=np.float32)))
        self.pack()


class Surrogate:
    """Ensemble of networks plus the normalization they were trained with."""

    def __init__(self, members: int = 4, device=0, seed: int = 0):
        torch = _torch()
        if not 1 <= members <= 8:
            raise ValueError("members must be in 1..8")
        self.device = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        L = lib()
        P, Pk = int(L.hadros_mlp_param_count()), int(L.hadros_mlp_packed_count())
        # the members' arrays stacked, so one call trains them side by side
        f32 = dict(dtype=torch.float32, device=self.device)
        self.stack = {"master": torch.empty((members, P), **f32), "m": torch.empty((members, P), **f32),
                      "v": torch.empty((members, P), **f32), "grad": torch.empty((members, P), **f32),
                      "packed": torch.empty((members, Pk), dtype=torch.bfloat16, device=self.device)}
        self.nets = [Network(self.device, seed * 1000 + k, {key: t[k] for key, t in self.stack.items()})
                     for k in range(members)]
        self.norm: HadrosMlpNorm | None = None
        self.seed = seed
        self._images = None
        self.history: list[list[float]] = []

    # ---- features -----------------------------------------------------------
    def featurize(self, raw, stream=None):
        torch = _torch()
        X = torch.empty((raw.shape[0], N_INPUT), dtype=torch.bfloat16, device=self.device)
        _check(lib().hadros_mlp_featurize(_vp(raw), int(raw.shape[0]), C.byref(self.norm), _vp(X),
                                          _stream_ptr(stream)))
        return X

    def standardize(self, targets):
        torch = _torch()
        mu = torch.tensor([self.norm.out_mu[o] for o in range(N_OUT)], device=self.device)
        sd = torch.tensor([self.norm.out_sd[o] for o in range(N_OUT)], device=self.device)
        return ((targets - mu) / sd).float().contiguous()

    # ---- training -----------------------------------------------------------
    def fit(self, raw, targets, epochs: int = 20, batch: int = 8192, lr: float = 2e-3,
            lr_min: float = 2e-5, weight=None, floors=(TAU_FLOOR, 0.0),
            log_every: int = 0, graph: bool = True) -> list[list[float]]:
        """Train every member on (raw features, ln targets) with Adam and a cosine
        learning rate; the members see the data in different orders and step
        together.  graph=True: the steps run from a CUDA graph that holds a
        group of training steps (hadros_mlp_train_members_dev, whose step
        counter and schedule live on the device), replayed through each
        epoch; graph=False: one hadros_mlp_train_members call per step."""
        torch = _torch()
        L = lib()
        if self.norm is None:
            self.norm = make_norm(raw, targets, floors)
        X = self.featurize(raw)
        T = self.standardize(targets)
        W = None if weight is None else weight.float().contiguous()
        n = int(raw.shape[0])
        K = len(self.nets)
        batch = min(batch, n)
        steps_per_epoch = max(n // batch, 1)
        total = steps_per_epoch * epochs
        ws = torch.empty(int(L.hadros_mlp_members_workspace_bytes(K, batch)), dtype=torch.uint8, device=self.device)
        idx = torch.empty((K, n), dtype=torch.int64, device=self.device)
        loss = torch.zeros(K, dtype=torch.float32, device=self.device)
        gens = []
        for k in range(K):
            g = torch.Generator(device=self.device)
            g.manual_seed(self.seed * 7919 + k)
            gens.append(g)
        st = self.stack
        step = self.nets[0].step
        Wp = None if W is None else _vp(W)
        graph_obj, group = None, 1
        if graph:
            group = max(d for d in range(1, min(64, steps_per_epoch) + 1) if steps_per_epoch % d == 0)
            sched = abi.HadrosTrainSched(lr, lr_min, 0.9, 0.999, 1e-8, step + total, steps_per_epoch)
            step_dev = torch.full((1,), step, dtype=torch.int64, device=self.device)

            def call(arrays, counter, stream):
                _check(L.hadros_mlp_train_members_dev(
                    K, batch, _vp(X), _vp(T), Wp, _vp(idx), n, _vp(arrays["master"]), _vp(arrays["packed"]),
                    _vp(arrays["m"]), _vp(arrays["v"]), _vp(arrays["grad"]), C.byref(sched), _vp(counter), _vp(ws),
                    _vp(loss), C.c_void_p(stream.cuda_stream)))
            # one call on copies loads the kernels before the capture
            idx.copy_(torch.arange(n, device=self.device).expand(K, n))
            call({k: t.clone() for k, t in st.items()}, torch.zeros(1, dtype=torch.int64, device=self.device),
                 torch.cuda.current_stream(self.device))
            torch.cuda.synchronize(self.device)
            cap = torch.cuda.Stream(device=self.device)
            cap.wait_stream(torch.cuda.current_stream(self.device))
            graph_obj = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph_obj, stream=cap):
                for _ in range(group):
                    call(st, step_dev, cap)
        sp = _stream_ptr(None)
        self.history = [[] for _ in range(K)]
        for ep in range(epochs):
            for k in range(K):
                idx[k] = torch.randperm(n, device=self.device, generator=gens[k])
            loss.zero_()
            if graph_obj is not None:
                for _ in range(steps_per_epoch // group):
                    graph_obj.replay()
                step += steps_per_epoch
            else:
                for b in range(steps_per_epoch):
                    t = step / max(total - 1, 1)
                    opt = HadrosAdam(lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * t)), 0.9, 0.999, 1e-8)
                    step += 1
                    _check(L.hadros_mlp_train_members(
                        K, batch, _vp(X), _vp(T), Wp, C.c_void_p(idx.data_ptr() + 8 * b * batch), n,
                        _vp(st["master"]), _vp(st["packed"]), _vp(st["m"]), _vp(st["v"]), _vp(st["grad"]),
                        C.byref(opt), step, _vp(ws), _vp(loss), sp))
            lv = (loss / steps_per_epoch).tolist()
            if any(math.isnan(x) for x in lv):
                raise HadrosError(abi.E_TIMEOUT, "NaN training loss: a tensor-core kernel timed out or training diverged")
            for k in range(K):
                self.history[k].append(lv[k])
            if log_every and (ep + 1) % log_every == 0:
                print(f"epoch {ep + 1}: loss " + " ".join(f"{x:.3e}" for x in lv), flush=True)
        del graph_obj
        for net in self.nets:
            net.step = step
        self._images = None
        return self.history

    # ---- inference ----------------------------------------------------------
    def forward(self, raw, batch: int = 65536):
        """ln tau_E, ln I_E of every member for raw feature rows: [members][n][2]
        (through the training forward kernels)."""
        torch = _torch()
        X = self.featurize(raw)
        n = int(raw.shape[0])
        bs = min(batch, n)
        ws = torch.empty(int(lib().hadros_mlp_workspace_bytes(bs)), dtype=torch.uint8, device=self.device)
        res = torch.empty((len(self.nets), n, N_OUT), dtype=torch.float32, device=self.device)
        mu = torch.tensor([self.norm.out_mu[o] for o in range(N_OUT)], device=self.device)
        sd = torch.tensor([self.norm.out_sd[o] for o in range(N_OUT)], device=self.device)
        st = _stream_ptr(None)
        for k, net in enumerate(self.nets):
            for a in range(0, n, bs):
                b = min(n, a + bs)
                xb = X[a:b].contiguous()
                ob = torch.empty((b - a, N_OUT), dtype=torch.float32, device=self.device)
                _check(lib().hadros_mlp_forward(_vp(net.master), _vp(net.packed), _vp(xb), b - a, _vp(ws),
                                                _vp(ob), st))
                res[k, a:b] = ob * sd + mu
        return res

    def _weights(self):
        torch = _torch()
        if self._images is None:
            L = lib()
            nb = int(L.hadros_mlp_image_bytes())
            K = len(self.nets)
            self._masters = self.stack["master"]
            self._images = torch.empty(K * nb, dtype=torch.uint8, device=self.device)
            for k, net in enumerate(self.nets):
                _check(L.hadros_mlp_pack_image(_vp(net.packed), C.c_void_p(self._images.data_ptr() + k * nb),
                                               _stream_ptr(None)))
        return self._masters, self._images

    def image(self, p, sigma, pixel_begin: int = 0, pixel_end: int | None = None, threshold: float = 0.01,
              per_bin: bool = True, stream=None, out: dict | None = None, spread_of: int = 0) -> dict:
        """Surrogate image of pixels [pixel_begin, pixel_end) on the GPU.  Returns
        device tensors (ln_tau_E, ln_I_E per bin when per_bin; tau, P_surv, I_obs,
        spread per pixel; fallback_ids, counters) without synchronizing.  The
        spread is over ln I_obs (spread_of 0) or ln tau (spread_of 1)."""
        torch = _torch()
        P = int(p.nx) * int(p.ny)
        pe = P if pixel_end is None else int(pixel_end)
        n, B = pe - int(pixel_begin), n_bins_of(p)
        masters, images = self._weights()
        if out is None:
            out = alloc_image(n, B, self.device, per_bin)
        o = HadrosSurrogateOut()
        for key in ("ln_tau_E", "ln_I_E", "tau", "P_surv", "I_obs", "spread", "fallback_ids", "counters"):
            t = out.get(key)
            setattr(o, key, None if t is None else t.data_ptr())
        _check(lib().hadros_surrogate_image(C.byref(p), sigma.handle, len(self.nets), _vp(masters), _vp(images),
                                            C.byref(self.norm), int(pixel_begin), pe, float(threshold),
                                            int(spread_of), C.byref(o), _stream_ptr(stream)))
        return out

    def image_with_fallback(self, ctx, p, sigma, threshold: float = 0.01, spread_of: int = 0) -> dict:
        """Surrogate image whose flagged pixels are replaced by the exact tracer.
        Host numpy arrays; 'fallback' holds the traced pixel ids."""
        torch = _torch()
        res = self.image(p, sigma, threshold=threshold, per_bin=False, spread_of=spread_of)
        torch.cuda.synchronize(self.device)
        cnt = res["counters"].cpu().numpy()
        if cnt[1]:
            raise HadrosError(abi.E_TIMEOUT, "surrogate inference kernel timed out")
        ids = np.sort(res["fallback_ids"][:int(cnt[0])].cpu().numpy())
        img = {k: res[k].cpu().numpy() for k in ("tau", "P_surv", "I_obs", "spread")}
        if ids.size:
            ex = ctx.image(p, sigma, pixel_ids=ids, outputs=("tau", "P_surv", "I_obs"))
            for k in ("tau", "P_surv", "I_obs"):
                img[k][ids] = ex[k]
        img["fallback"] = ids
        return img

    # ---- persistence --------------------------------------------------------
    def save(self, path) -> None:
        nm = self.norm
        np.savez(path, masters=np.stack([net.master.cpu().numpy() for net in self.nets]),
                 feat_mu=np.array(nm.feat_mu[:]), feat_inv_sd=np.array(nm.feat_inv_sd[:]),
                 out_mu=np.array(nm.out_mu[:]), out_sd=np.array(nm.out_sd[:]),
                 out_floor=np.array(nm.out_floor[:]))

    @classmethod
    def load(cls, path, device=0) -> "Surrogate":
        d = np.load(path)
        sur = cls(members=int(d["masters"].shape[0]), device=device)
        for net, m in zip(sur.nets, d["masters"]):
            net.load_master(m)
        nm = HadrosMlpNorm()
        for key in ("feat_mu", "feat_inv_sd", "out_mu", "out_sd", "out_floor"):
            arr = getattr(nm, key)
            for i, v in enumerate(d[key]):
                arr[i] = float(v)
        sur.norm = nm
        return sur


def alloc_image(n_pixels: int, n_bins: int, device, per_bin: bool = True) -> dict:
    torch = _torch()
    f32, f64 = torch.float32, torch.float64
    out = {"tau": torch.empty(n_pixels, dtype=f64, device=device),
           "P_surv": torch.empty(n_pixels, dtype=f64, device=device),
           "I_obs": torch.empty(n_pixels, dtype=f64, device=device),
           "spread": torch.empty(n_pixels, dtype=f32, device=device),
           "fallback_ids": torch.empty(max(n_pixels, 1), dtype=torch.int32, device=device),
           "counters": torch.zeros(2, dtype=torch.int32, device=device)}
    if per_bin:
        out["ln_tau_E"] = torch.empty((n_pixels, n_bins), dtype=f32, device=device)
        out["ln_I_E"] = torch.empty((n_pixels, n_bins), dtype=f32, device=device)
    return out


def raw_features(p, sigma, pixel_ids, device=0):
    """Raw features [len(pixel_ids) * B][16] of a camera's samples (device)."""
    torch = _torch()
    ids = torch.as_tensor(np.ascontiguousarray(pixel_ids, dtype=np.int32), device=device)
    B = n_bins_of(p)
    raw = torch.empty((ids.numel() * B, N_FEATURES), dtype=torch.float32, device=device)
    _check(lib().hadros_mlp_raw_features(C.byref(p), sigma.handle, _vp(ids), int(ids.numel()), _vp(raw),
                                         _stream_ptr(None)))
    return raw


def targets_of(tau_E, I_E, i_floor: float):
    """ln(tau_E + TAU_FLOOR), ln(I_E + i_floor) as float32 [n][2] (numpy in)."""
    t = np.log(np.asarray(tau_E, dtype=np.float64).reshape(-1) + TAU_FLOOR)
    i = np.log(np.asarray(I_E, dtype=np.float64).reshape(-1) + i_floor)
    return np.stack([t, i], axis=1).astype(np.float32)


def trace_samples(ctx, sigma, cams, pixels_per_cam: int, seed: int = 20261203, device=0,
                  i_floor: float | None = None, chunk: int = 64):
    """Training samples traced by the exact tracer: for each camera a seeded
    random pixel subset, all of its bins, `chunk` cameras per launch
    (hadros_batch_pixels).  Returns (raw [n][16], ln targets [n][2]) as device
    tensors and a dict with the floor and tracing time."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    raws, taus, Is = [], [], []
    t0 = time.perf_counter()
    for a in range(0, len(cams), chunk):
        part = cams[a:a + chunk]
        lists = []
        for p in part:
            P = int(p.nx) * int(p.ny)
            lists.append(np.sort(rng.choice(P, size=min(pixels_per_cam, P), replace=False)).astype(np.int32))
        res = ctx.batch_pixels(part, sigma, lists, outputs=("tau_E", "I_E"))
        for p, ids, r in zip(part, lists, res):
            taus.append(r["tau_E"].reshape(-1))
            Is.append(r["I_E"].reshape(-1))
            raws.append(raw_features(p, sigma, ids, device))
    torch.cuda.synchronize(device)
    t_trace = time.perf_counter() - t0
    tau = np.concatenate(taus)
    I = np.concatenate(Is)
    if i_floor is None:
        i_floor = float(I.max()) * I_FLOOR_REL if I.max() > 0 else 1e-300
    y = torch.from_numpy(targets_of(tau, I, i_floor)).to(device)
    return torch.cat(raws), y, {"i_floor": i_floor, "trace_s": t_trace, "n": int(tau.size)}


def time_fit(rows: int = 1 << 20, epochs: int = 2, batch: int = 8192, members: int = 4, device: int = 0) -> dict:
    """Seconds per training step of an ensemble of `members` networks on
    `rows` synthetic samples (16 raw features with a one-hot profile block,
    two smooth targets): one warm-up epoch (kernel loading, graph capture),
    then `epochs` timed epochs."""
    torch = _torch()
    torch.cuda.set_device(device)
    rng = np.random.default_rng(1)
    raw = rng.normal(size=(rows, 16)).astype(np.float32)
    raw[:, 5:13] = 0.0
    raw[np.arange(rows), 5 + rng.integers(0, 8, rows)] = 1.0
    y = np.stack([np.sin(raw[:, 0]) + raw[:, 15], raw[:, 1] * raw[:, 2]], axis=1).astype(np.float32)
    sur = Surrogate(members=members, device=device, seed=1)
    R = torch.from_numpy(raw).to(sur.device)
    Y = torch.from_numpy(y).to(sur.device)
    sur.fit(R, Y, epochs=1, batch=batch)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sur.fit(R, Y, epochs=epochs, batch=batch)
    torch.cuda.synchronize()
    steps = epochs * max(rows // batch, 1)
    return {"rows": rows, "epochs": epochs, "batch": batch, "members": members, "steps": steps,
            "s_per_step": (time.perf_counter() - t0) / steps, "loss": [h[-1] for h in sur.history]}


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="time the ensemble's training step on synthetic rows")
    ap.add_argument("--rows", type=int, default=1 << 20)
    ap.add_argument("--epochs", type=int, default=2)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--members", type=int, default=4)
    a = ap.parse_args()
    print(json.dumps(time_fit(a.rows, a.epochs, a.batch, a.members)))
