"""Surrogate-accelerated parameter scans, timed against the plain tracer.

    python -m hadros_b200.scan production --points 256 --side 4096 --bins 64
    torchrun --nproc-per-node N -m hadros_b200.scan production ...   # points split over N GPUs
    python -m hadros_b200.scan inference            # 2048^2 x 32 with fallback
    python -m hadros_b200.scan batched              # 64 cameras, one graph-captured launch

production: the surrogate is trained on rays the tracer traces at other
parameter points of the same box (collapsar_ndaf_like, density_weighted
source, a = 0.95, rho0 log-uniform in [1e9, 1e12], inclination in [10, 80]
deg); each scan point is then evaluated by the ensemble, the pixels whose
ensemble standard deviation of ln I_obs exceeds a threshold (chosen on
held-out cameras so that pixels below it err by more than the --bound
rarely, or --bound / --sigmas) are traced exactly, and the exact tracer
judges a seeded random 1% of the pixels.  The plain tracer's time per
point is measured on a few points of the same scan.

batched: 64 cameras of uneven size (64..1024 pixels a side), spin,
inclination, all eight profiles and rho0, 16 bins, traced in one persistent
launch from an autotuned plan replayed from a CUDA graph, against the same
cameras traced one launch each.

learning-curve: the configuration-4 general model's held-out error against
its training-set size, for one ensemble over all profiles and one per
profile kind.

inference: the surrogate is trained on cameras with randomized spin,
inclination, profile, rho0 and two shape parameters, and evaluates the
mixed_512 camera at 2048 x 2048 x 32 bins with exact fallback.

Prints one JSON object.  Everything runs on CUDA device 0.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import Context, SigmaTable, n_bins_of, params, spectral_bins
from . import surrogate as S
from . import workloads as W


def _torch():
    import torch
    return torch


def plain_image(ctx, p, sigma) -> tuple[dict, float]:
    """The exact tracer's per-pixel outputs in device memory (the current
    device), and its time (s)."""
    torch = _torch()
    P = int(p.nx) * int(p.ny)
    dev = torch.device("cuda", torch.cuda.current_device())
    out = {"tau": torch.empty(P, dtype=torch.float64, device=dev),
           "P_surv": torch.empty(P, dtype=torch.float64, device=dev),
           "I_obs": torch.empty(P, dtype=torch.float64, device=dev),
           "fate": torch.empty(P, dtype=torch.int8, device=dev),
           "steps": torch.empty(P, dtype=torch.int32, device=dev)}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.image_device(p, sigma, out, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    return out, time.perf_counter() - t0


def errors(I_ex: np.ndarray, I_sur: np.ndarray, floor_rel: float = 1e-6) -> dict:
    """Relative errors over the pixels whose exact value is at least floor_rel
    of the largest judged value (intensity, or optical depth)."""
    I_ex = np.asarray(I_ex, dtype=np.float64)
    I_sur = np.asarray(I_sur, dtype=np.float64)
    top = float(I_ex.max()) if I_ex.size else 0.0
    m = I_ex >= floor_rel * top if top > 0 else np.zeros(I_ex.shape, bool)
    if not m.any():
        return {"n": 0, "worst": 0.0, "p99": 0.0, "median": 0.0}
    rel = np.abs(I_sur[m] - I_ex[m]) / I_ex[m]
    return {"n": int(m.sum()), "worst": float(rel.max()), "p99": float(np.quantile(rel, 0.99)),
            "median": float(np.median(rel))}


CANDIDATE_THRESHOLDS = (0.002, 0.0025, 0.0033, 0.004, 0.005, 0.0067, 0.01)
# Escalation schedule of a scan point whose exact judge finds an error above
# the bound: the spread thresholds tried in turn (on the 256-point production
# scan, 4 points judged above 1 % at 0.01 and none at 0.0033).
ESCALATE = (0.005, 0.0033, 0.002)


def judge_ids(P: int, frac: float, rng) -> np.ndarray:
    """A seeded random judge subset: round(frac P) distinct pixel ids (int32)."""
    n = max(1, int(round(frac * P)))
    return rng.choice(P, size=n, replace=False).astype(np.int32)


class PointRunner:
    """Scan points evaluated on one device with buffers allocated once.

    run() enqueues, on `stream`: the ensemble's image of the camera (the
    inference kernel, which lists the pixels whose spread exceeds the
    threshold), then ONE exact trace of the judge pixels followed by the
    fallback pixels (the fallback ids land right after the judge ids in one
    device list), then the fallback pixels' exact values into the image.  It
    waits on the stream for the fallback count and for the judged errors it
    returns."""

    KEYS = ("tau", "P_surv", "I_obs")

    def __init__(self, ctx, sigma, sur, side: int, n_bins: int, judge_frac: float = 0.01, stream=None):
        torch = _torch()
        self.ctx, self.sigma, self.sur = ctx, sigma, sur
        self.P = side * side
        self.n_judge = max(1, int(round(judge_frac * self.P)))
        dev = sur.device
        self.stream = stream
        # judge ids, then room for every pixel as a fallback
        self.ids = torch.empty(self.n_judge + self.P, dtype=torch.int32, device=dev)
        self.out = S.alloc_image(self.P, n_bins, dev, per_bin=False)
        del self.out["fallback_ids"]
        self.out["fallback_ids"] = self.ids[self.n_judge:]
        self.exact = {k: torch.empty(self.n_judge + self.P, dtype=torch.float64, device=dev) for k in self.KEYS}

    def run(self, p, threshold: float, jids, spread_of: int = 0, detail: bool = False, escalate=(),
            bound: float | None = None) -> dict:
        """One scan point.  jids: the judge pixel ids (device int32 tensor of
        n_judge, or host array).  Returns host values: fallback count, judged
        errors, device times of the parts (ms).

        escalate: lower spread thresholds tried in turn while the judged worst
        error exceeds `bound`; each traces exactly only the pixels whose spread
        lies between the new and the previous threshold and replaces them (the
        spread does not always flag the rare pixels a point gets wrong, and the
        exact judge is what shows it)."""
        torch = _torch()
        st = self.stream if self.stream is not None else torch.cuda.current_stream()
        nj = self.n_judge
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        with torch.cuda.stream(st):
            if isinstance(jids, np.ndarray):
                jids = torch.from_numpy(np.ascontiguousarray(jids, dtype=np.int32)).to(self.ids.device)
            if jids.data_ptr() != self.ids.data_ptr():
                self.ids[:nj].copy_(jids, non_blocking=True)
            ev[0].record(st)
            self.sur.image(p, self.sigma, threshold=threshold, per_bin=False, out=self.out, stream=st,
                           spread_of=spread_of)
            ev[1].record(st)
            cnt = self.out["counters"].cpu()        # waits for the inference kernel
            if int(cnt[1]):
                raise RuntimeError("surrogate inference kernel timed out")
            nf = int(cnt[0])
            jt = self.ids[:nj].long()
            raw = {k: self.out[k][jt] for k in self.KEYS}   # surrogate values before the fallback
            spread_j = self.out["spread"][jt]
            self.ctx.pixels_device(p, self.sigma, self.ids, self.exact, n=nj + nf, stream=st)
            ev[2].record(st)
            if nf:
                fb = self.ids[nj:nj + nf].long()
                for k in self.KEYS:
                    self.out[k].index_copy_(0, fb, self.exact[k][nj:nj + nf])
            key = "I_obs" if spread_of == 0 else "tau"
            ex = self.exact[key][:nj]
            e_all = _device_errors(ex, self.out[key][jt])
            fbmask = torch.zeros(nj, dtype=torch.bool, device=ex.device)
            if nf:
                # judged pixels that fell back hold exact values; the surrogate's own errors exclude them
                fbmask = torch.isin(self.ids[:nj], self.ids[nj:nj + nf])
            e_sur = _device_errors(ex[~fbmask], raw[key][~fbmask])
            pmax = (self.exact["P_surv"][:nj] - self.out["P_surv"][jt]).abs().max()
            ev[3].record(st)
            vals = torch.stack([*e_all, *e_sur, pmax.double()]).cpu()      # waits for the step
        v = vals.numpy().copy()
        esc_thr, n_esc = threshold, 0
        if escalate and bound is not None and v[1] > bound:
            with torch.cuda.stream(st):
                sp = self.out["spread"]
                for thr2 in sorted(escalate, reverse=True):
                    if thr2 >= esc_thr:
                        continue
                    ids2 = torch.nonzero((sp > thr2) & (sp <= esc_thr)).flatten().to(torch.int32)
                    n2 = int(ids2.numel())
                    esc_thr = thr2
                    if n2:
                        o = nj + nf + n_esc
                        self.ids[o:o + n2].copy_(ids2)
                        self.ctx.pixels_device(p, self.sigma, self.ids[o:o + n2],
                                               {k: self.exact[k][o:o + n2] for k in self.KEYS}, stream=st)
                        fb2 = self.ids[o:o + n2].long()
                        for k in self.KEYS:
                            self.out[k].index_copy_(0, fb2, self.exact[k][o:o + n2])
                        n_esc += n2
                    pm2 = (self.exact["P_surv"][:nj] - self.out["P_surv"][jt]).abs().max().double()
                    e2 = torch.stack([*_device_errors(ex, self.out[key][jt]), pm2]).cpu().numpy()
                    v[0:4] = e2[:4]
                    v[8] = e2[4]
                    if v[1] <= bound:
                        break
        nf_all = nf + n_esc
        res = {"fallback_pixels": nf_all, "fallback_frac": nf_all / self.P, "judged": nj, "judged_quantity": key,
               "threshold_used": esc_thr, "escalated_pixels": n_esc,
               "error": {"n": int(v[0]), "worst": float(v[1]), "p99": float(v[2]), "median": float(v[3])},
               "error_surrogate_pixels": {"n": int(v[4]), "worst": float(v[5]), "p99": float(v[6]),
                                          "median": float(v[7])},
               "P_surv_max_abs_error": float(v[8]),
               "inference_ms": ev[0].elapsed_time(ev[1]), "exact_ms": ev[1].elapsed_time(ev[2]),
               "device_ms": ev[0].elapsed_time(ev[3])}
        if detail:
            res["judge"] = {"ids": self.ids[:nj].cpu().numpy(), "spread": spread_j.cpu().numpy(),
                            "exact": {k: self.exact[k][:nj].cpu().numpy() for k in self.KEYS},
                            "raw": {k: t.cpu().numpy() for k, t in raw.items()}}
        return res

    def alloc_host(self) -> dict:
        """Pinned host buffers for run_host: the judge ids and the image."""
        torch = _torch()
        h = {k: torch.empty(self.P, dtype=torch.float64, pin_memory=True) for k in self.KEYS}
        h["judge_ids"] = torch.empty(self.n_judge, dtype=torch.int32, pin_memory=True)
        return h

    def run_host(self, p, threshold: float, host: dict, spread_of: int = 0, escalate=(),
                 bound: float | None = None) -> dict:
        """run() from host memory to host memory: the judge ids in
        host["judge_ids"] go to the device, the finished image (tau, P_surv,
        I_obs) comes back into host[...]; returns run()'s dict plus the bytes
        copied each way."""
        torch = _torch()
        st = self.stream if self.stream is not None else torch.cuda.current_stream()
        with torch.cuda.stream(st):
            self.ids[:self.n_judge].copy_(host["judge_ids"], non_blocking=True)
            res = self.run(p, threshold, self.ids[:self.n_judge], spread_of=spread_of, escalate=escalate,
                           bound=bound)
            for k in self.KEYS:
                host[k].copy_(self.out[k], non_blocking=True)
            st.synchronize()
        # judge ids and the exact trace's camera tables in; the image, the
        # fallback count and the judged errors out
        res["h2d_bytes"] = self.n_judge * 4 + int(self.ctx.stats()["h2d_bytes"])
        res["d2h_bytes"] = 8 * self.P * len(self.KEYS) + 8 + 9 * 8
        return res


def _device_errors(ex, got, floor_rel: float = 1e-6):
    """(n, worst, p99, median) of |got - ex| / ex over the pixels with ex at
    least floor_rel of the largest ex, as 0-d device tensors (zeros if none)."""
    torch = _torch()
    z = torch.zeros((), dtype=torch.float64, device=ex.device)
    if ex.numel() == 0:
        return z, z, z, z
    top = ex.max()
    m = (ex >= floor_rel * top) & (top > 0)
    rel = torch.where(m, (got - ex).abs() / torch.where(m, ex, torch.ones_like(ex)), torch.zeros_like(ex))
    n = m.sum().double()
    worst = rel.max().double()
    # quantiles over the kept pixels: the others sort below every kept one
    srt = torch.sort(torch.where(m, rel, torch.full_like(rel, -1.0))).values
    k0 = rel.numel() - m.sum()

    def q(f):
        idx = (k0 + (f * (n - 1)).floor().long()).clamp(0, rel.numel() - 1)
        return torch.where(n > 0, srt[idx].double(), z)
    return n, worst, q(0.99), q(0.5)


def surrogate_point(ctx, sigma, sur, p, threshold: float, judge_frac: float, rng, buf=None,
                    spread_of: int = 0, escalate=(), bound: float | None = None) -> dict:
    """One scan point: surrogate image, exact fallback, exact judge subset
    (PointRunner), with its wall-clock time.

    Besides the errors of the result, reports for other spread thresholds what
    they would have given: the fraction of pixels above them and the worst
    judged error among the pixels below them (the surrogate's values there).
    `buf`: a PointRunner to reuse (else one is made for this camera)."""
    torch = _torch()
    if int(p.nx) != int(p.ny):
        raise ValueError("scan points are square images")
    P = int(p.nx) * int(p.ny)
    runner = buf if isinstance(buf, PointRunner) else PointRunner(ctx, sigma, sur, int(p.nx), n_bins_of(p),
                                                                  judge_frac)
    jids = judge_ids(P, judge_frac, rng)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = runner.run(p, threshold, jids, spread_of=spread_of, detail=True, escalate=escalate, bound=bound)
    t_total = time.perf_counter() - t0
    jd = res.pop("judge")
    key = res["judged_quantity"]
    sj = jd["spread"]
    sp = runner.out["spread"]
    what_if = []
    for thr in CANDIDATE_THRESHOLDS:
        keep = sj <= thr
        e = errors(jd["exact"][key][keep], jd["raw"][key][keep]) if keep.any() else {"worst": 0.0, "n": 0}
        what_if.append({"threshold": thr, "fallback_frac": float((sp > thr).float().mean().item()),
                        "worst": e["worst"], "n": e["n"]})
    res.update({"seconds": t_total, "inference_s": res["inference_ms"] / 1e3,
                "exact_s": t_total - res["inference_ms"] / 1e3,
                "spread_quantiles": [float(q) for q in np.quantile(sj, [0.5, 0.9, 0.99, 0.999])],
                "what_if": what_if})
    return res


def production_cam(rho0: float, theta_deg: float, side: int, n_bins: int):
    return params(**W.production_point(nx=side, ny=side, rho0_gcm3=rho0, theta_obs_deg=theta_deg,
                                       n_bins=n_bins))


def n_held_out(n_cams: int, val_frac: float = 0.1) -> int:
    return max(1, int(round(val_frac * n_cams)))


def held_out_samples(ctx, sigma, cams, pixels_per_cam: int, seed: int, i_floor: float, device=0):
    """The held-out cameras' samples (the last n_held_out cameras), as train() traces them."""
    n_val = n_held_out(len(cams))
    vraw, vy, _ = S.trace_samples(ctx, sigma, cams[-n_val:], pixels_per_cam, seed=seed + 1, i_floor=i_floor,
                                  device=device)
    return cams[-n_val:], vraw, vy


def calibrate(sur, sigma, cams, raw, y, i_floor: float, bound: float, q: float = 0.99, margin: float = 0.8,
              floor_rel: float = 1e-6) -> dict:
    """The spread threshold, chosen on held-out cameras.

    For every held-out pixel (all its bins are in raw/y, camera by camera):
    the ensemble's I_obs as the inference kernel forms it (log-sum-exp over the
    bins of the members' mean ln I_E + ln dE), its relative error against the
    traced I_obs, and the spread (standard deviation over members of each
    member's ln I_obs).  The threshold is the largest one (on a log grid from
    bound/30 to bound) for which, among the pixels above floor_rel of the
    brightest whose spread is at most the threshold, no more than a fraction
    1 - q err by more than margin x bound.  The tail this admits is the scan's
    per-point escalation's job (PointRunner.run): a point whose exact judge
    finds an error above the bound lowers its threshold."""
    torch = _torch()
    B = n_bins_of(cams[0])
    bins = spectral_bins(cams[0], sigma)
    valid = (np.asarray(bins["valid"]) != 0) & (np.asarray(bins["dE"]) > 0)
    dE = torch.tensor(np.where(valid, bins["dE"], 0.0), dtype=torch.float64, device=raw.device)
    lnde = torch.tensor(np.where(valid, np.log(np.where(valid, bins["dE"], 1.0)), -np.inf),
                        dtype=torch.float64, device=raw.device)
    fw = sur.forward(raw).double()                      # [K][n][2]
    K, n = fw.shape[0], fw.shape[1]
    P = n // B
    lnI = fw[:, :, 1].reshape(K, P, B)
    L_k = torch.logsumexp(lnI + lnde, dim=2)            # [K][P]
    spread = L_k.std(0, unbiased=False)
    I_sur = torch.exp(torch.logsumexp(lnI.mean(0) + lnde, dim=1))
    I_ex = ((torch.exp(y[:, 1].double()) - i_floor).clamp_min(0.0).reshape(P, B) * dE).sum(1)
    m = I_ex >= floor_rel * I_ex.max()
    err = ((I_sur - I_ex).abs() / I_ex)[m].cpu().numpy()
    sp = spread[m].cpu().numpy()
    bad = err > margin * bound
    chosen = bound / 30.0
    for t in np.geomspace(bound / 30.0, bound, 61):
        keep = sp <= t
        if keep.any() and bad[keep].mean() > 1.0 - q:
            break
        chosen = float(t)
    return {"threshold": chosen, "q": q, "margin": margin, "pixels": int(m.sum().item()),
            "error_p99": float(np.quantile(err, 0.99)), "error_max": float(err.max()),
            "spread_median": float(np.median(sp)), "fallback_frac_held_out": float((sp > chosen).mean())}


def train(ctx, sigma, cams, pixels_per_cam: int, members: int, epochs: int, seed: int, batch: int,
          lr: float, device=0) -> tuple[object, dict]:
    """Trace training samples on `cams`, hold out the last cameras
    (n_held_out), train the ensemble; returns it with timing and validation RMS."""
    torch = _torch()
    n_val = n_held_out(len(cams))
    raw, y, info = S.trace_samples(ctx, sigma, cams[:-n_val], pixels_per_cam, seed=seed, device=device)
    _, vraw, vy = held_out_samples(ctx, sigma, cams, pixels_per_cam, seed, info["i_floor"], device)
    sur = S.Surrogate(members=members, device=device, seed=seed)
    t0 = time.perf_counter()
    sur.fit(raw, y, epochs=epochs, batch=batch, lr=lr, floors=(S.TAU_FLOOR, info["i_floor"]))
    torch.cuda.synchronize()
    t_fit = time.perf_counter() - t0
    pred = sur.forward(vraw).mean(0)
    d = (pred - vy).double()
    rms = torch.sqrt((d ** 2).mean(0)).cpu().numpy()
    info.update(fit_s=t_fit, samples=int(raw.shape[0]), val_samples=int(vraw.shape[0]),
                val_rms_ln_tau=float(rms[0]), val_rms_ln_I=float(rms[1]),
                final_loss=[h[-1] for h in sur.history])
    return sur, info


def save_model(path, sur, info: dict) -> None:
    """The ensemble (npz) and its training record (json beside it)."""
    sur.save(path)
    with open(str(path) + ".json", "w") as f:
        json.dump(info, f, default=float)


def load_model(path, device=0) -> tuple[object, dict]:
    sur = S.Surrogate.load(path, device)
    with open(str(path) + ".json") as f:
        info = json.load(f)
    info["loaded_from"] = str(path)
    return sur, info


def run_points(n_points: int, evaluate, dist=None, rank: int = 0, world: int = 1) -> list | None:
    """Scan points 0..n_points-1 split over the ranks (equal cost each,
    hadros_b200.shard.run_scan): this rank evaluates its points with
    `evaluate(k) -> row`; rank 0 returns every row in point order, the
    others None."""
    from . import shard
    return shard.run_scan(list(range(n_points)), lambda ks: [evaluate(k) for k in ks], dist, rank, world,
                          costs=[1.0] * n_points)


def point_rng(k: int):
    """The judge subset's generator of scan point k (independent of which
    rank evaluates the point)."""
    return np.random.default_rng([W.SEED + 5, k])


def run_production(a) -> dict | None:
    """The production scan on this process's GPU, or under torchrun on every
    rank's GPU with the scan points split over the ranks (each rank trains
    the same ensemble from the same seeds; rows meet on rank 0)."""
    from . import shard
    torch = _torch()
    dist, rank, world, local = shard.init_from_env()
    E, g2, s = W.synthetic_sigma_arrays()
    sigma = SigmaTable.from_arrays(E, s, g2)
    try:
        with Context(local) as ctx:
            tpts = W.scan_points(a.train_points, seed=W.SEED + 17)
            cams = [production_cam(r, t, a.train_side, a.bins) for r, t in tpts]
            if a.load:
                sur, info = load_model(a.load, local)
            else:
                sur, info = train(ctx, sigma, cams, a.pixels_per_cam, a.members, a.epochs, W.SEED, a.batch, a.lr,
                                  device=local)
                if a.save and rank == 0:
                    save_model(a.save, sur, info)
            calib = None
            if a.sigmas <= 0:   # calibrated bound: c x spread, c from the held-out cameras
                vcams, vraw, vy = held_out_samples(ctx, sigma, cams, a.pixels_per_cam, W.SEED, info["i_floor"],
                                                   local)
                calib = calibrate(sur, sigma, vcams, vraw, vy, info["i_floor"], a.bound)
                a.threshold = calib["threshold"]
                if rank == 0:
                    print(json.dumps({"calibration": calib}), file=sys.stderr, flush=True)
            pts = W.scan_points(a.points, seed=W.SEED)
            buf = PointRunner(ctx, sigma, sur, a.side, a.bins, a.judge)

            def evaluate(k):
                r, t = pts[k]
                row = surrogate_point(ctx, sigma, sur, production_cam(r, t, a.side, a.bins), a.threshold,
                                      a.judge, point_rng(k), buf, escalate=a.escalate, bound=a.bound)
                row["point"] = k
                print(json.dumps({"point": k, "rank": rank, "seconds": row["seconds"],
                                  "fallback_frac": row["fallback_frac"], "worst": row["error"]["worst"],
                                  "p99": row["error"]["p99"], "threshold_used": row["threshold_used"]}),
                      file=sys.stderr, flush=True)
                return row
            t0 = time.perf_counter()
            rows = run_points(len(pts), evaluate, dist, rank, world)
            scan_wall = time.perf_counter() - t0
            del buf
            plain = []
            if rank == 0:
                for r, t in pts[:a.plain_points]:
                    _, sec = plain_image(ctx, production_cam(r, t, a.side, a.bins), sigma)
                    plain.append(sec)
                    torch.cuda.empty_cache()
    finally:
        if dist is not None:
            dist.destroy_process_group()
    if rows is None:
        return None
    sur_total = sum(x["seconds"] for x in rows)
    plain_per_point = float(np.mean(plain)) if plain else float("nan")
    setup = info["trace_s"] + info["fit_s"]
    n_full = a.scan_total or len(rows)
    sur_per_point = sur_total / len(rows)
    return {
        "workload": "production_scan", "points": a.points, "side": a.side, "bins": a.bins, "ranks": world,
        "members": a.members, "bound": a.bound, "sigmas": a.sigmas, "threshold": a.threshold,
        "calibration": calib, "judge_frac": a.judge,
        "train": info,
        "surrogate_s_per_point": sur_total / len(rows),
        "scan_wall_s": scan_wall,
        "plain_s_per_point": plain_per_point,
        "speedup_scan": plain_per_point * len(rows) / (sur_total + setup),
        "scan_total_points": n_full,
        "speedup_full_scan": plain_per_point * n_full / (setup + n_full * sur_per_point),
        "speedup_per_point": plain_per_point * len(rows) / sur_total,
        "fallback_frac_mean": float(np.mean([x["fallback_frac"] for x in rows])),
        "fallback_frac_max": float(np.max([x["fallback_frac"] for x in rows])),
        "worst_pixel_error": max(x["error"]["worst"] for x in rows),
        "escalate": list(a.escalate),
        "points_escalated": sum(1 for x in rows if x["escalated_pixels"] > 0),
        "p99_error_max": max(x["error"]["p99"] for x in rows),
        "median_error_mean": float(np.mean([x["error"]["median"] for x in rows])),
        "per_point": rows,
    }


def run_inference(a) -> dict:
    torch = _torch()
    E, g2, s = W.synthetic_sigma_arrays()
    sigma = SigmaTable.from_arrays(E, s, g2)
    with Context(0) as ctx:
        cams = [params(**c) for c in W.surrogate_training_cams(a.train_points, side=a.train_side, n_bins=a.bins)]
        sur, info = train(ctx, sigma, cams, a.pixels_per_cam, a.members, a.epochs, W.SEED, a.batch, a.lr)
        p = params(**W.surrogate_inference_image(nx=a.side, ny=a.side, n_bins=a.bins))
        row = surrogate_point(ctx, sigma, sur, p, a.threshold, a.judge, np.random.default_rng(W.SEED + 9),
                              spread_of=1)
        _, sec = plain_image(ctx, p, sigma)
        del torch
    return {"workload": "surrogate_inference", "side": a.side, "bins": a.bins, "members": a.members,
            "train": info, "surrogate": row, "plain_s": sec, "speedup": sec / row["seconds"]}


def _held_out_rms(sur, raw, y) -> list[float]:
    torch = _torch()
    d = (sur.forward(raw).mean(0) - y).double()
    return torch.sqrt((d ** 2).mean(0)).cpu().tolist()


def run_learning_curve(a) -> dict:
    """The general model of the configuration-4 surrogate (spin, inclination,
    all eight profiles, rho0 and two shape parameters randomized): held-out
    RMS of ln tau_E and ln I_E against the number of training samples, for
    one ensemble over all profiles and for one ensemble per profile kind
    (trained on that kind's cameras only), and the share of the inference
    image's pixels above the calibrated 1% threshold for each."""
    torch = _torch()
    E, g2, s = W.synthetic_sigma_arrays()
    sigma = SigmaTable.from_arrays(E, s, g2)
    out = {"workload": "learning_curve", "bins": a.bins, "members": a.members, "epochs": a.epochs,
           "pixels_per_cam": a.pixels_per_cam, "general": [], "per_profile": {}}
    with Context(0) as ctx:
        kws = W.surrogate_training_cams(a.train_points, side=a.train_side, n_bins=a.bins)
        cams = [params(**c) for c in kws]
        n_val = n_held_out(len(cams))
        train_cams, val_cams = cams[:-n_val], cams[-n_val:]
        raw, y, info = S.trace_samples(ctx, sigma, train_cams, a.pixels_per_cam, seed=W.SEED)
        vraw, vy, _ = S.trace_samples(ctx, sigma, val_cams, a.pixels_per_cam, seed=W.SEED + 1,
                                      i_floor=info["i_floor"])
        per_cam = a.pixels_per_cam * a.bins
        p_inf = params(**W.surrogate_inference_image(nx=a.side, ny=a.side, n_bins=a.bins))
        for frac in (0.25, 0.5, 1.0):
            n = int(len(train_cams) * frac) * per_cam
            sur = S.Surrogate(members=a.members, seed=W.SEED)
            t0 = time.perf_counter()
            sur.fit(raw[:n], y[:n], epochs=a.epochs, batch=a.batch, lr=a.lr, floors=(S.TAU_FLOOR, info["i_floor"]))
            torch.cuda.synchronize()
            row = {"samples": n, "fit_s": time.perf_counter() - t0, "val_rms": _held_out_rms(sur, vraw, vy)}
            if frac == 1.0:
                res = sur.image(p_inf, sigma, threshold=0.01 / 3.0, per_bin=False, spread_of=1)
                torch.cuda.synchronize()
                row["inference_fallback_frac"] = int(res["counters"][0].item()) / (a.side * a.side)
            out["general"].append(row)
            print(json.dumps({"general": row}), file=sys.stderr, flush=True)
        # one ensemble per profile kind
        kinds = [int(c.profile_kind) for c in cams]
        se = [0.0, 0.0]
        nv = 0
        for kind in range(8):
            tr = [i for i, c in enumerate(train_cams) if int(c.profile_kind) == kind]
            va = [i for i, c in enumerate(val_cams) if int(c.profile_kind) == kind]
            if not tr:
                continue
            idx = torch.cat([torch.arange(i * per_cam, (i + 1) * per_cam, device=raw.device) for i in tr])
            sur = S.Surrogate(members=a.members, seed=W.SEED + kind)
            sur.fit(raw[idx], y[idx], epochs=a.epochs, batch=a.batch, lr=a.lr, floors=(S.TAU_FLOOR, info["i_floor"]))
            row = {"train_cams": len(tr), "val_cams": len(va)}
            if va:
                vidx = torch.cat([torch.arange(i * per_cam, (i + 1) * per_cam, device=raw.device) for i in va])
                rms = _held_out_rms(sur, vraw[vidx], vy[vidx])
                row["val_rms"] = rms
                for o in range(2):
                    se[o] += rms[o] ** 2 * vidx.numel()
                nv += vidx.numel()
            if kind == int(p_inf.profile_kind):
                res = sur.image(p_inf, sigma, threshold=0.01 / 3.0, per_bin=False, spread_of=1)
                torch.cuda.synchronize()
                row["inference_fallback_frac"] = int(res["counters"][0].item()) / (a.side * a.side)
            out["per_profile"][hb_profile_name(kind)] = row
            print(json.dumps({"profile": kind, **row}), file=sys.stderr, flush=True)
        out["per_profile_val_rms"] = [float(np.sqrt(x / max(nv, 1))) for x in se]
        del kinds
    return out


def hb_profile_name(kind: int) -> str:
    from . import lib
    name = lib().hadros_profile_name(kind)
    return name.decode() if name else str(kind)


def run_batched(a) -> dict:
    """The batched scan: every camera in one persistent launch from a plan
    whose schedule the autotuner picked, captured in a CUDA graph and
    replayed; against the same cameras traced one launch after another."""
    torch = _torch()
    from . import autotune as AT
    E, g2, s = W.synthetic_sigma_arrays()
    sigma = SigmaTable.from_arrays(E, s, g2)
    cams = [params(**c) for c in W.batched_scan(a.points)]
    dev = torch.device("cuda", 0)
    P = sum(int(c.nx) * int(c.ny) for c in cams)
    B = n_bins_of(cams[0])
    with Context(0) as ctx:
        t0 = time.perf_counter()
        sched, rep = AT.autotune(ctx, cams, sigma, torch, scale=8, repeats=1, use_cache=False)
        t_tune = time.perf_counter() - t0
        t0 = time.perf_counter()
        plan = ctx.plan(cams, sigma, sched)
        t_plan = time.perf_counter() - t0
        out = plan.alloc(torch, device=dev, outputs=("tau", "P_surv", "I_obs", "fate", "steps"))
        st = torch.cuda.Stream()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=st):
            plan.launch(out, st)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        with torch.cuda.stream(st):
            g.replay()
        e1.record(st)
        torch.cuda.synchronize()
        t_graph = e0.elapsed_time(e1) / 1e3
        steps_graph = int(out["steps"].to(torch.int64).sum().item())
        del g
        plan.close()
        # the same cameras, one launch each (the reference's per-camera loop)
        pmax = max(int(c.nx) * int(c.ny) for c in cams)
        one = {"tau": torch.empty(pmax, dtype=torch.float64, device=dev),
               "P_surv": torch.empty(pmax, dtype=torch.float64, device=dev),
               "I_obs": torch.empty(pmax, dtype=torch.float64, device=dev),
               "fate": torch.empty(pmax, dtype=torch.int8, device=dev),
               "steps": torch.empty(pmax, dtype=torch.int32, device=dev)}
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for c in cams:
            ctx.image_device(c, sigma, one, stream=torch.cuda.current_stream())
        torch.cuda.synchronize()
        t_sep = time.perf_counter() - t0
    return {"workload": "batched_scan", "cameras": len(cams), "pixels": P, "bins": B,
            "schedule": rep["best"], "autotune_s": t_tune, "plan_s": t_plan,
            "graph_replay_s": t_graph, "pixel_bins_per_s": P * B / t_graph,
            "separate_launches_s": t_sep, "speedup_vs_separate": t_sep / t_graph,
            "accepted_steps": steps_graph, "autotune": rep["timings"]}


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("workload", choices=("production", "inference", "batched", "learning-curve"))
    ap.add_argument("--points", type=int, default=256)
    ap.add_argument("--scan-total", type=int, default=0,
                    help="points of the whole scan when --points runs its first ones (for the "
                         "extrapolated speedup; 0 = --points)")
    ap.add_argument("--plain-points", type=int, default=2)
    ap.add_argument("--side", type=int, default=None)
    ap.add_argument("--bins", type=int, default=None)
    ap.add_argument("--train-points", type=int, default=128)
    ap.add_argument("--train-side", type=int, default=4096)
    ap.add_argument("--pixels-per-cam", type=int, default=1024)
    ap.add_argument("--members", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--bound", type=float, default=0.01,
                    help="relative error bound above which a pixel is traced exactly")
    ap.add_argument("--sigmas", type=float, default=0.0,
                    help="fallback above bound / sigmas ensemble standard deviations; 0 (default, "
                         "production): a threshold chosen on the held-out cameras")
    ap.add_argument("--judge", type=float, default=0.01)
    ap.add_argument("--escalate", default=",".join(str(x) for x in ESCALATE),
                    help="production: lower spread thresholds tried in turn at a point whose judged worst "
                         "error exceeds the bound (comma-separated; empty: none)")
    ap.add_argument("--save", default=None, help="write the trained ensemble here (npz + json)")
    ap.add_argument("--load", default=None, help="use an ensemble written by --save instead of training")
    a = ap.parse_args(argv)
    a.escalate = tuple(float(x) for x in a.escalate.split(",") if x.strip())
    a.threshold = a.bound / (a.sigmas if a.sigmas > 0 else 3.0)
    if a.workload == "production":
        a.side = a.side or 4096
        a.bins = a.bins or 64
        out = run_production(a)
    elif a.workload == "learning-curve":
        a.side = a.side or 2048
        a.bins = a.bins or 32
        out = run_learning_curve(a)
    elif a.workload == "batched":
        a.points = a.points if a.points != 256 else 64
        out = run_batched(a)
    else:
        a.side = a.side or 2048
        a.bins = a.bins or 32
        out = run_inference(a)
    if out is not None:
        print(json.dumps(out, default=float))


if __name__ == "__main__":
    main()
