#!/usr/bin/env python
"""bench.py — pixel-bins/s of the HADROS per-pixel image pipeline on B200.

Default workload (the production scan, 4096 x 4096 pixels x 64 bins): a step
is one parameter point of the scan evaluated by the learned surrogate with
its exact-tracer fallback and a seeded random 1% of the pixels judged by the
exact tracer (hadros_b200.scan.PointRunner).  The ensemble is trained before
the timed region on rays the tracer traces at other points of the same
parameter box; the plain tracer (every pixel exact) is timed once on one
point beside it.  One process per GPU; each GPU evaluates its own scan
points (no data-path collective: weak scaling).

  value        device-timed throughput of the steps (CUDA events, max over
               ranks), outputs resident in HBM
  e2e          the same steps from host memory to host memory
               (PointRunner.run_host: judge ids in, the image out)
  roofline     the trace kernel's FP64 rate on the plain-tracer point against
               the measured FP64 peak (cuBLAS DGEMM in the same run);
               roofline_inference: the surrogate kernel against BF16 peak
  cpu_baseline the reference CPU code on the host cores over a strided pixel
               sample of a scan point (every pixel traced exactly, as the
               reference does)

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --workload image       # the 512x512x8 mixed image, trace kernel only
    python bench.py --workload surrogate   # the surrogate's tcgen05 inference kernel
    python bench.py --mev                  # image workload with the MeV thermal channel
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

# Algorithmic FP64 work, counted from the reference formulas with their
# duplicate inverse-metric evaluations removed (+,-,*,/ = 1 flop; FMA = 2;
# transcendentals not counted): one RKF45 attempt = 6 RHS (192 each) + stage
# inputs + y4/y5 + error = 1573 flop; one accepted step's ZAMO interval and
# redshift = 52 flop.  Per point 44 flop and per point-bin 16 flop of transfer.
F_ATT, F_GEO, F_PT, F_PB = 1573, 52, 44, 16
# The MeV thermal channel (physical model, default profiles, monochromatic),
# FP64 per path point: interval in cm 1, density 30, redshift 1, temperature 3,
# electron fraction 6, local energy 1, opacity 24, emissivity 31, transfer 12.
F_MEV = 109
FP64_PEAK_DATASHEET_TFLOPS = 37.0
WORKLOAD_DESC = ("512x512 px x 8 powerlaw_cutoff bins (1e5-1e12 GeV), a=0.998, i=17 deg, "
                 "powerlaw_funnel_envelope, funnel_wall source, r_obs 60 M, fov 25 deg, h0 0.01, "
                 "FP64 RKF45 geodesics + FP32 Kahan transfer")


def env_int(name: str, default: int) -> int:
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


# --------------------------------------------------------------------------- CPU baseline

def cpu_sample(params_kw: dict, stride: int, threads: int, mev_off: bool = False) -> dict:
    """Time the reference CPU implementation (oracle/_ref, or the oracle port)
    on every `stride`-th pixel in i and j of the image.  The reference always
    runs its MeV block; mev_off=True gives it the cheapest setting the CPU app
    accepts (MEV_MODEL toy with URCA, pair, bremsstrahlung, absorption and
    scattering off: apps/compute_kerr_image_from_cache.cpp argv 45-51)."""
    import hadros_b200 as hb
    from hadros_b200 import workloads as W
    from oracle import pyoracle as O
    E, g2, s = W.synthetic_sigma_arrays()
    kw = dict(params_kw)
    if mev_off:
        kw.update(mev_channel=1, mev_model="toy", mev_urca=False, mev_pair=False, mev_brems=False,
                  mev_absorption=False, mev_scattering=False)
    p = hb.params(**kw)
    ids = W.strided_pixels(p.nx, p.ny, stride)
    B = 1 if p.spectral_kind == 0 else p.n_bins
    kind = "reference" if O.ref_available() else "port"
    t0 = time.perf_counter()
    if kind == "reference":
        O.ref_image(p, E, g2, s, pixel_ids=ids, threads=threads, per_bin=False)
    else:
        O.oracle_image(p, E, s, pixel_ids=ids, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": ids.size * B / dt, "seconds": dt, "rays": int(ids.size), "kind": kind,
            "cores": threads, "stride": stride, "mev_off": mev_off}


def describe_cpu(c: dict, nx: int, ny: int) -> str:
    what = ("reference CPU code built from its sources (KerrCamera::trace_pixel + "
            "integrate_kerr_ray_spectral, MeV block as shipped)" if c["kind"] == "reference"
            else "CPU oracle port (oracle/hadros_oracle.c)")
    return (f"every {c['stride']}th pixel in i and j of the {nx}x{ny} image ({c['rays']} rays), "
            f"{what}, OpenMP {c['cores']} threads, {c['seconds']:.1f} s")


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_arm(args) -> None:
    """--impl reference: the reference's own CPU implementation on the host cores."""
    rank = env_int("RANK", 0)
    if rank != 0:
        return
    from hadros_b200 import workloads as W
    kw = W.mixed_512()
    threads = host_threads()
    stride = 48
    for _ in range(args.warmup):
        cpu_sample(kw, stride, threads)
    times, last = [], None
    for _ in range(args.steps):
        last = cpu_sample(kw, stride, threads)
        times.append(last["seconds"])
    per_step = sum(times) / len(times)
    value = last["rays"] * kw["n_bins"] / per_step
    off = cpu_sample(kw, stride, threads, mev_off=True)
    line = {
        "impl": "reference", "metric": "pixel-bins/sec", "value": value, "unit": "pixel-bins/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "mixed_512: " + WORKLOAD_DESC,
                   "sample": f"every {stride}th pixel in i and j ({last['rays']} rays) per step"},
        "cpu_baseline": {"value": value, "unit": "pixel-bins/s", "cores": threads,
                         "kind": last["kind"], "sample": describe_cpu(last, 512, 512),
                         "value_mev_off": off["value"],
                         "mev_off": "the same sample with the MeV block at its cheapest setting "
                                    "(toy model, five terms off)"},
        "e2e": {"value": value, "unit": "pixel-bins/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def reference_cuda_arm(args) -> None:
    """--impl reference-cuda: the reference's own GPU executable
    (apps/compute_kerr_image_cuda.cu, built from its source by
    oracle/build_ref.sh into oracle/_ref/compute_kerr_image_cuda) on the bench
    camera with a monochromatic 1e9 GeV spectrum (the only kind it traces), next
    to this library on the same image.  The reference runs twice: with its
    Makefile launch settings (32x32 tiles, 128 steps per launch,
    Makefile:208-209; at most 64x64 pixels, as that setting leaves all but 8 SMs
    idle and needs minutes per 256x256 image) and with the whole image as one
    tile and 1024 steps per launch, its best setting; its RKF45 tolerance is
    set to the CPU image path's 1e-6, which this library uses.  Its own
    printed timing is used (host clock around its tile loop and file writes,
    rays/s).  Rank 0 only."""
    import torch

    import hadros_b200 as hb
    from hadros_b200 import workloads as W
    if env_int("RANK", 0) != 0:
        return
    exe = ROOT / "oracle" / "_ref" / "compute_kerr_image_cuda"
    side = args.side or 256
    kw = W.mixed_512(nx=side, ny=side, spectral="monochromatic", Enu_obs_GeV=1.0e9)
    if not exe.exists():
        print(json.dumps({"impl": "reference-cuda", "unavailable": "oracle/_ref/compute_kerr_image_cuda not built"}))
        return
    E, g2, s = W.synthetic_sigma_arrays()
    f = lambda x: f"{x:.17g}"   # noqa: E731
    argv = [f(kw["Enu_obs_GeV"]), f(kw["a_spin"]), f(kw["M_bh_msun"]), f(kw["rho0_gcm3"]), f(kw["r0_rg"]),
            f(kw["sigma_r_rg"]), f(kw["H_over_R"]), f(kw["src_r_center_rg"]), f(kw["src_sigma_r_rg"]),
            f(kw["src_theta_width_deg"]), f(kw["src_powerlaw"]), f(kw["src_emax_GeV"]), f(kw["src_norm"]),
            "10", "1", f(kw["theta_obs_deg"]), f(kw["r_obs_rg"]), f(kw["fov_deg"]), str(side), str(side),
            f(kw["r_max_rg"]), f(kw["h"])]
    tail = ["200000", "1e-6", "powerlaw_funnel_envelope", f(kw["radial_power"]), f(kw["funnel_depletion"]),
            f(kw["funnel_theta_deg"]), f(kw["envelope_rho0_gcm3"]), f(kw["envelope_alpha"]),
            f(kw["torus_r_min_rg"]), f(kw["torus_r_max_rg"]), f(kw["rho_floor_gcm3"]), "funnel_wall",
            f(kw["src_funnel_theta_deg"]), "1", "2", "0.1", "1", "-1", "0", "100"]
    runs = {}
    with tempfile.TemporaryDirectory() as td:
        Path(td, "data", "sigma").mkdir(parents=True)
        Path(td, "output", "images").mkdir(parents=True)
        W.write_sigma_file(Path(td, "data", "sigma", "sigma_nuN_CC_GBW.dat"), E, g2, s)
        small = min(side, 64)
        for name, n, tile, spl in ((f"makefile_tiles_32_steps_128_{small}x{small}", small, 32, 128),
                                   (f"one_tile_steps_1024_{side}x{side}", side, side, 1024)):
            a = list(argv)
            a[18] = a[19] = str(n)
            r = subprocess.run([str(exe), *a, str(tile), str(spl), *tail], cwd=td, capture_output=True,
                               text=True, timeout=1200)
            line = next((ln for ln in r.stdout.splitlines() if ln.startswith("CUDA timing:")), "")
            if r.returncode != 0 or not line:
                runs[name] = {"failed": (r.stderr or r.stdout)[-300:]}
                continue
            parts = line.split()
            runs[name] = {"seconds": float(parts[2]), "rays_per_s": float(parts[4]),
                          "accepted_steps": int(line.rsplit("=", 1)[1]),
                          "advance_launches": int(line.split("advance launches=")[1].split(",")[0])}
    # this library on the same image (device-timed; default fast arithmetic)
    sig = hb.SigmaTable.from_arrays(E, s, g2)
    ours = {}
    with hb.Context(0) as ctx:
        for prec in ("fp64", "mixed"):
            p = hb.params(**dict(kw, precision=prec))
            ctx.image(p, sig, outputs=("steps",))            # warm-up
            img = ctx.image(p, sig, outputs=("steps",))
            st = ctx.stats()
            ours[prec] = {"seconds": st["kernel_ms"] / 1e3, "rays_per_s": side * side / (st["kernel_ms"] / 1e3),
                          "e2e_seconds": st["total_ms"] / 1e3, "accepted_steps": int(img["steps"].sum())}
    line = {"impl": "reference-cuda", "metric": "rays/sec", "unit": "rays/s",
            "config": {"workload": f"mixed_512 camera at {side}x{side}, monochromatic 1e9 GeV, "
                                   "powerlaw_funnel_envelope, funnel_wall, RKF45 tol 1e-6"},
            "reference_cuda": runs, "hadros_b200": ours,
            "gpu": torch.cuda.get_device_name(0)}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- production scan

SCAN_DESC = ("production scan, one parameter point per step: 4096x4096 px x 64 powerlaw_cutoff bins "
             "(1e5-1e12 GeV, gamma 2, Ecut 1e12), collapsar_ndaf_like (r0 12, sigma_r 8, H 0.45, r 3-80), "
             "density_weighted source, a=0.95, rho0 log-uniform 1e9-1e12, inclination U[10,80] deg, "
             "r_obs 60 M, fov 25 deg, h0 0.01; surrogate (4-network BF16 ensemble) + exact fallback + "
             "exact judge of a seeded random 1% of pixels per point; exact tracer FP64 RKF45 geodesics + "
             "FP32 Kahan transfer")
SCAN_SIDE, SCAN_BINS, SCAN_POINTS = 4096, 64, 256
REF_GRID = 15          # reference sample per step: a 15 x 15 strided grid of pixels


def scan_config(world: int) -> dict:
    return {"workload": SCAN_DESC, "side": SCAN_SIDE, "bins": SCAN_BINS,
            "l2": "image outputs (403 MB) larger than L2, and a 256 MiB write between steps",
            "parallelism": f"scan points split over {world} GPU(s), no collective on the data path"}


def scan_point_kw(k: int) -> dict:
    """Camera keywords of scan point k (of SCAN_POINTS, seeded)."""
    from hadros_b200 import workloads as W
    rho0, theta = W.scan_points(SCAN_POINTS)[k % SCAN_POINTS]
    return W.production_point(nx=SCAN_SIDE, ny=SCAN_SIDE, n_bins=SCAN_BINS, rho0_gcm3=rho0,
                              theta_obs_deg=theta)


def ref_sample_ids(k: int, grid: int = REF_GRID, side: int = SCAN_SIDE) -> np.ndarray:
    """Step k's reference sample: a grid x grid strided pixel set whose offset
    moves with k, so the steps' samples are disjoint."""
    stride = side // grid
    oi, oj = (k * 37) % stride, (k * 101) % stride
    ii = oi + stride * np.arange(grid)
    jj = oj + stride * np.arange(grid)
    return (jj[:, None] * side + ii[None, :]).ravel().astype(np.int32)


def cpu_scan_sample(k: int, threads: int, grid: int = REF_GRID, mev_off: bool = False) -> dict:
    """The reference CPU code (oracle/_ref, else the oracle port) on step k's
    sample of scan point k: every pixel exact, all bins, MeV block as shipped
    (or at its cheapest setting with mev_off)."""
    import hadros_b200 as hb
    from hadros_b200 import workloads as W
    from oracle import pyoracle as O
    E, g2, s = W.synthetic_sigma_arrays()
    kw = scan_point_kw(k)
    if mev_off:
        kw.update(mev_channel=1, mev_model="toy", mev_urca=False, mev_pair=False, mev_brems=False,
                  mev_absorption=False, mev_scattering=False)
    p = hb.params(**kw)
    ids = ref_sample_ids(k, grid)
    kind = "reference" if O.ref_available() else "port"
    t0 = time.perf_counter()
    if kind == "reference":
        r = O.ref_image(p, E, g2, s, pixel_ids=ids, threads=threads, per_bin=False)
    else:
        r = O.oracle_image(p, E, s, pixel_ids=ids, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": ids.size * SCAN_BINS / dt, "seconds": dt, "rays": int(ids.size), "kind": kind,
            "cores": threads, "steps_per_ray": float(np.mean(r["steps"])), "point": k % SCAN_POINTS}


def reference_scan_arm(args) -> None:
    """--impl reference on the scan workload: the reference computes every
    pixel of a scan point exactly (it has no surrogate); each step times its
    CPU code on a different strided sample of a different point (ref_grid^2
    rays, disjoint across steps), with all host threads."""
    if env_int("RANK", 0) != 0:
        return
    threads = host_threads()
    for w in range(args.warmup):        # untimed: small samples of the warm-up points
        cpu_scan_sample(w, threads, grid=2)
    g = args.ref_grid
    rows = [cpu_scan_sample(args.warmup + k, threads, grid=g) for k in range(args.steps)]
    per_step = sum(r["seconds"] for r in rows) / len(rows)
    value = g * g * SCAN_BINS / per_step
    off = cpu_scan_sample(args.warmup, threads, grid=g, mev_off=True)
    kind = rows[0]["kind"]
    sample = (f"{len(rows)} steps x {g}x{g} strided pixels (stride {SCAN_SIDE // g}, "
              f"offset moving per step: {len(rows) * g * g} distinct rays) of scan points "
              f"{args.warmup}..{args.warmup + len(rows) - 1}, all {SCAN_BINS} bins, "
              + ("reference CPU code built from its sources (KerrCamera::trace_pixel + "
                 "integrate_kerr_ray_spectral, MeV block as shipped)" if kind == "reference"
                 else "CPU oracle port (oracle/hadros_oracle.c)") + f", OpenMP {threads} threads")
    line = {
        "impl": "reference", "metric": "pixel-bins/sec", "value": value, "unit": "pixel-bins/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": scan_config(args.gpus),
        "cpu_baseline": {"value": value, "unit": "pixel-bins/s", "cores": threads, "kind": kind,
                         "sample": sample, "rays": len(rows) * g * g,
                         "steps_per_ray": float(np.mean([r["steps_per_ray"] for r in rows])),
                         "value_mev_off": off["value"],
                         "mev_off": "step 0's sample with the MeV block at its cheapest setting "
                                    "(toy model, five terms off)"},
        "e2e": {"value": value, "unit": "pixel-bins/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-i", str(self.idx), "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        self.file.flush()
        rows = []
        try:
            text = Path(self.file.name).read_text()
            for r in csv.reader(io.StringIO(text)):
                if len(r) >= 9:
                    rows.append([x.strip() for x in r])
        finally:
            os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "", 1).isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "", 1).isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        load = sorted(sm)[len(sm) // 4:] if sm else []
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(rows)}


# --------------------------------------------------------------------------- GPU arm

def fp64_peak_tflops(torch, device) -> float:
    """cuBLAS DGEMM 8192^3 on this GPU, best of 5 (CUDA events)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def read_traffic() -> tuple[float | None, str | None]:
    """DRAM bytes per trace-kernel launch from a committed ncu summary."""
    f = ROOT / "profiles" / "ncu_traffic.json"
    if not f.exists():
        return None, None
    d = json.loads(f.read_text())
    return d.get("bytes_per_launch"), d.get("source")


def read_traffic_per_step() -> tuple[float | None, str | None]:
    """DRAM bytes per accepted step of the production trace kernel (deferred
    transfer, 64 bins) from a committed ncu summary of a 256x256 launch."""
    f = ROOT / "profiles" / "ncu_traffic_production.json"
    if not f.exists():
        return None, None
    d = json.loads(f.read_text())
    return d.get("bytes_per_accepted_step"), d.get("source")


def gpu_arm(args) -> None:
    import torch

    import hadros_b200 as hb
    from hadros_b200 import workloads as W

    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=device)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    kw = W.mixed_512(**({"mev_channel": 1} if args.mev else {}))
    p = hb.params(**kw)          # library default: fast geodesic arithmetic
    E, g2, s = W.synthetic_sigma_arrays()
    sig = hb.SigmaTable.from_arrays(E, s, g2)
    ctx = hb.Context(local)
    P, B = p.nx * p.ny, p.n_bins
    f32 = p.precision == hb.PRECISION_MIXED
    out = {
        "tau": torch.empty(P, dtype=torch.float64, device=device),
        "P_surv": torch.empty(P, dtype=torch.float64, device=device),
        "I_obs": torch.empty(P, dtype=torch.float64, device=device),
        "fate": torch.empty(P, dtype=torch.int8, device=device),
        "steps": torch.empty(P, dtype=torch.int32, device=device),
        "attempts": torch.empty(P, dtype=torch.int32, device=device),
        "tau_E": torch.empty(P * B, dtype=torch.float32 if f32 else torch.float64, device=device),
        "I_E": torch.empty(P * B, dtype=torch.float64, device=device),
    }
    if args.mev:
        out.update({k: torch.empty(P, dtype=torch.float64, device=device) for k in hb.MEV_OUTPUTS})
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)   # > 126 MB L2
    # a non-default stream: the library launches on it, the events bracket it
    stream = torch.cuda.Stream(device=device)
    torch.cuda.set_stream(stream)

    for _ in range(args.warmup):
        ctx.image_device(p, sig, out, stream)
        flush.zero_()
    ctx.synchronize()
    barrier()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    gpu_index = local
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        try:
            gpu_index = int(vis.split(",")[local])
        except (ValueError, IndexError):
            gpu_index = local
    launches = 0
    with ClockSampler(gpu_index) as clocks:
        t_start.record(stream)
        for k in range(args.steps):
            ev[k][0].record(stream)
            ctx.image_device(p, sig, out, stream)
            launches += ctx.stats()["launches"]
            ev[k][1].record(stream)
            flush.zero_()
        t_end.record(stream)
        torch.cuda.synchronize()
        barrier()
    clk = clocks.summary()
    ctx.synchronize()
    elapsed = t_start.elapsed_time(t_end) / 1e3
    kernel_ms = [a.elapsed_time(b) for a, b in ev]
    elapsed_max = max_over_ranks(elapsed)
    per_step = elapsed_max / args.steps
    value = world * P * B / per_step

    attempts = float(out["attempts"].to(torch.int64).sum().item())
    steps_sum = float(out["steps"].to(torch.int64).sum().item())
    flop64 = attempts * F_ATT + steps_sum * (F_GEO + (F_MEV if args.mev else 0))
    flop32 = steps_sum * (F_PT + B * F_PB)
    kern_s = statistics.mean(kernel_ms) / 1e3
    peak = fp64_peak_tflops(torch, device)
    achieved = flop64 / kern_s / 1e12
    traffic, traffic_src = read_traffic()

    # e2e through the C-ABI call with host buffers (hadros_image)
    barrier()
    t0 = time.perf_counter()
    h2d = d2h = 0
    e2e_kernel_ms = []
    for _ in range(args.steps):
        ctx.image(p, sig)
        st = ctx.stats()
        h2d, d2h = st["h2d_bytes"], st["d2h_bytes"]
        e2e_kernel_ms.append(st["kernel_ms"])
    e2e_s = max_over_ranks(time.perf_counter() - t0) / args.steps
    e2e_value = world * P * B / e2e_s

    fates = torch.bincount(out["fate"].to(torch.int64), minlength=3).tolist()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        c = cpu_sample(kw, 24, host_threads())
        cpu = {"value": c["value"], "unit": "pixel-bins/s", "cores": c["cores"], "kind": c["kind"],
               "sample": describe_cpu(c, p.nx, p.ny)}
        if not args.mev and c["kind"] == "reference":   # the like-for-like figure for a UHE-only GPU line
            cpu["value_mev_off"] = cpu_sample(kw, 24, host_threads(), mev_off=True)["value"]
            cpu["mev_off"] = ("the same sample with the reference's MeV block at its cheapest setting "
                              "(toy model, five terms off)")
    total_steps = sum_over_ranks(steps_sum)
    if rank == 0:
        line = {
            "metric": "pixel-bins/sec", "value": value, "unit": "pixel-bins/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64+f32", "data": "synthetic",
            "config": {"workload": "mixed_512: " + WORKLOAD_DESC +
                                   (" + FP64 MeV thermal channel (physical, defaults)" if args.mev else ""),
                       "per_gpu": "one 512x512x8 image per GPU per step",
                       "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"independent images, {world} GPU(s), no collective"},
            "rays_per_s": world * P / per_step,
            "accepted_steps_per_s": total_steps / per_step,
            "fates": {"escaped": fates[0], "captured": fates[1], "truncated": fates[2]},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 "
                                        f"(datasheet {FP64_PEAK_DATASHEET_TFLOPS} TFLOP/s)",
                         "flop64_per_launch": flop64, "flop32_per_launch": flop32,
                         "kernel_ms": statistics.mean(kernel_ms),
                         "traffic": traffic, "traffic_source": traffic_src},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "pixel-bins/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3,
                    "kernel_ms": statistics.mean(e2e_kernel_ms)},
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def _dist_setup(torch, device, world: int, timeout_s: int):
    """NCCL process group (world > 1) and the barrier / max / sum helpers."""
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s), device_id=device)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def reduce(x: float, op: str) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
        return float(t.item())
    return dist, barrier, reduce


def gpu_index_of(local: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        try:
            return int(vis.split(",")[local])
        except (ValueError, IndexError):
            return local
    return local


def scan_arm(args) -> None:
    """The production scan: one surrogate-evaluated scan point per step."""
    import torch

    import hadros_b200 as hb
    from hadros_b200 import scan as SC
    from hadros_b200 import workloads as W

    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    # every rank trains its own copy of the ensemble (same seeds) before the
    # first collective, so no rank waits on another through the setup
    dist, barrier, reduce = _dist_setup(torch, device, world, 1800)
    E, g2, s = W.synthetic_sigma_arrays()
    sig = hb.SigmaTable.from_arrays(E, s, g2)
    ctx = hb.Context(local)
    P, B = SCAN_SIDE * SCAN_SIDE, SCAN_BINS

    # ---- setup (untimed): training rays, ensemble, fallback threshold ----------
    t_setup = time.perf_counter()
    tpts = W.scan_points(args.train_points, seed=W.SEED + 17)
    cams = [SC.production_cam(r, t, SCAN_SIDE, SCAN_BINS) for r, t in tpts]
    if args.model and os.path.exists(args.model):
        sur, info = SC.load_model(args.model, device=local)
    else:
        sur, info = SC.train(ctx, sig, cams, args.pixels_per_cam, 4, args.epochs, W.SEED, args.batch, args.lr,
                             device=local)
        if args.model and rank == 0:
            SC.save_model(args.model, sur, info)
    vcams, vraw, vy = SC.held_out_samples(ctx, sig, cams, args.pixels_per_cam, W.SEED, info["i_floor"], local)
    calib = SC.calibrate(sur, sig, vcams, vraw, vy, info["i_floor"], args.bound)
    del vraw, vy
    thr = calib["threshold"]
    setup_s = time.perf_counter() - t_setup

    stream = torch.cuda.Stream(device=device)
    torch.cuda.set_stream(stream)
    runner = SC.PointRunner(ctx, sig, sur, SCAN_SIDE, SCAN_BINS, args.judge, stream=stream)
    # this rank's scan points (every world-th), their judge subsets drawn ahead
    ks = [rank + world * k for k in range(args.warmup + args.steps)]
    pars = [hb.params(**scan_point_kw(k)) for k in ks]
    jrng = np.random.default_rng(W.SEED + 5 + rank)
    jids = [torch.from_numpy(SC.judge_ids(P, args.judge, jrng)).to(device) for _ in ks]
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)   # > 126 MB L2
    for w in range(args.warmup):
        runner.run(pars[w], thr, jids[w], escalate=SC.ESCALATE, bound=args.bound)
        flush.zero_()
    barrier()

    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rows = []
    with ClockSampler(gpu_index_of(local)) as clocks:
        t_start.record(stream)
        for k in range(args.steps):
            rows.append(runner.run(pars[args.warmup + k], thr, jids[args.warmup + k], escalate=SC.ESCALATE,
                                   bound=args.bound))
            flush.zero_()
        t_end.record(stream)
        torch.cuda.synchronize()
        barrier()
    clk = clocks.summary()
    elapsed = t_start.elapsed_time(t_end) / 1e3
    per_step = reduce(elapsed, "max") / args.steps
    value = world * P * B / per_step
    worst = reduce(max(r["error"]["worst"] for r in rows), "max")
    p99 = reduce(max(r["error"]["p99"] for r in rows), "max")
    fb_max = reduce(max(r["fallback_frac"] for r in rows), "max")
    inf_ms = statistics.mean(r["inference_ms"] for r in rows)
    ex_ms = statistics.mean(r["exact_ms"] for r in rows)

    # ---- the plain tracer on the last timed point: every pixel exact ----------
    k_plain = ks[args.warmup + args.steps - 1]
    pp = pars[args.warmup + args.steps - 1]
    plain = {"tau": torch.empty(P, dtype=torch.float64, device=device),
             "P_surv": torch.empty(P, dtype=torch.float64, device=device),
             "I_obs": torch.empty(P, dtype=torch.float64, device=device),
             "fate": torch.empty(P, dtype=torch.int8, device=device),
             "steps": torch.empty(P, dtype=torch.int32, device=device),
             "attempts": torch.empty(P, dtype=torch.int32, device=device)}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.image_device(pp, sig, plain, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_s = e0.elapsed_time(e1) / 1e3
    attempts = float(plain["attempts"].to(torch.int64).sum().item())
    steps_sum = float(plain["steps"].to(torch.int64).sum().item())
    flop64 = attempts * F_ATT + steps_sum * F_GEO
    peak64 = fp64_peak_tflops(torch, device)
    achieved = flop64 / plain_s / 1e12
    # the last step's finished image against the exact image, every pixel
    full = SC._device_errors(plain["I_obs"], runner.out["I_obs"])
    full_check = {"point": k_plain, "pixels": int(full[0].item()), "worst": float(full[1].item()),
                  "p99": float(full[2].item()), "median": float(full[3].item())}
    del plain
    bytes_per_accepted_step, traffic_src = read_traffic_per_step()
    traffic = bytes_per_accepted_step * steps_sum if bytes_per_accepted_step else None
    if traffic_src:
        traffic_src += " (bytes per accepted step of that launch x this launch's accepted steps)"

    # ---- e2e: the same steps from host memory to host memory --------------------
    host = runner.alloc_host()
    barrier()
    t0 = time.perf_counter()
    h2d = d2h = 0
    for k in range(args.steps):
        host["judge_ids"].copy_(jids[args.warmup + k].cpu())
        r = runner.run_host(pars[args.warmup + k], thr, host, escalate=SC.ESCALATE, bound=args.bound)
        h2d, d2h = r["h2d_bytes"], r["d2h_bytes"]
    e2e_s = reduce(time.perf_counter() - t0, "max") / args.steps
    del host

    # secondary key: the C2 image (mixed_512 camera, 512x512 x 8 bins), one
    # launch timed after a warm-up, outside the timed region
    c2 = None
    if rank == 0:
        p2 = hb.params(**W.mixed_512())
        P2, B2 = int(p2.nx) * int(p2.ny), int(p2.n_bins)
        o2 = {"tau": torch.empty(P2, dtype=torch.float64, device=device),
              "P_surv": torch.empty(P2, dtype=torch.float64, device=device),
              "I_obs": torch.empty(P2, dtype=torch.float64, device=device),
              "fate": torch.empty(P2, dtype=torch.int8, device=device),
              "steps": torch.empty(P2, dtype=torch.int32, device=device),
              "attempts": torch.empty(P2, dtype=torch.int32, device=device)}
        ctx.image_device(p2, sig, o2, stream)
        torch.cuda.synchronize()
        t2s = []
        for _ in range(2):
            e0.record(stream)
            ctx.image_device(p2, sig, o2, stream)
            e1.record(stream)
            torch.cuda.synchronize()
            t2s.append(e0.elapsed_time(e1) / 1e3)
        t2 = min(t2s)
        f2 = (float(o2["attempts"].to(torch.int64).sum().item()) * F_ATT
              + float(o2["steps"].to(torch.int64).sum().item()) * F_GEO)
        c2 = {"workload": "mixed_512: " + WORKLOAD_DESC, "value": P2 * B2 / t2, "unit": "pixel-bins/s",
              "ms_per_image": t2 * 1e3, "roofline_fp64": {"achieved": f2 / t2 / 1e12, "peak": peak64,
                                                          "frac": f2 / t2 / 1e12 / peak64}}
        del o2

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        c = cpu_scan_sample(k_plain, host_threads(), grid=args.cpu_grid)
        cpu = {"value": c["value"], "unit": "pixel-bins/s", "cores": c["cores"], "kind": c["kind"],
               "sample": (f"{c['rays']} pixels ({args.cpu_grid}x{args.cpu_grid} strided grid) of scan point "
                          f"{k_plain}, all {B} bins, every pixel exact, "
                          + ("reference CPU code built from its sources, MeV block as shipped"
                             if c["kind"] == "reference" else "CPU oracle port")
                          + f", OpenMP {c['cores']} threads, {c['seconds']:.1f} s"),
               "steps_per_ray_sample": c["steps_per_ray"],
               "steps_per_ray_gpu_image": steps_sum / P}
    peak16, peak16_src = measured_bf16_peak()
    inf_flop = P * B * len(sur.nets) * F_MLP
    if rank == 0:
        line = {
            "metric": "pixel-bins/sec", "value": value, "unit": "pixel-bins/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16+f64+f32",
            "data": "synthetic: seeded scan points; the ensemble is trained in this run (before the timed "
                    f"region) on rays the tracer traced at {args.train_points} other points of the box",
            "config": scan_config(world),
            "surrogate": {"worst_judged_error": worst, "p99_judged_error_max": p99,
                          "median_judged_error_mean": statistics.mean(r["error"]["median"] for r in rows),
                          "judged_pixels_per_point": rows[0]["judged"],
                          "fallback_frac_mean": statistics.mean(r["fallback_frac"] for r in rows),
                          "fallback_frac_max": fb_max, "threshold": thr, "bound": args.bound,
                          "escalate": list(SC.ESCALATE),
                          "steps_escalated": sum(1 for r in rows if r["escalated_pixels"] > 0),
                          "calibration": calib, "members": len(sur.nets),
                          "train": {k: info[k] for k in ("samples", "trace_s", "fit_s", "val_rms_ln_tau",
                                                         "val_rms_ln_I", "loaded_from") if k in info},
                          "epochs": args.epochs, "setup_s": setup_s},
            "plain_tracer": {"seconds_per_point": plain_s, "pixel_bins_per_s": P * B / plain_s,
                             "point": k_plain, "speedup_of_surrogate_step": plain_s / per_step,
                             "accepted_steps_per_ray": steps_sum / P, "full_image_check": full_check},
            "step_ms": {"inference": inf_ms, "exact_judge_and_fallback": ex_ms,
                        "rest": per_step * 1e3 - inf_ms - ex_ms},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                         "frac": achieved / peak64, "kernel": "trace kernel on the plain-tracer point",
                         "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 "
                                        f"(datasheet {FP64_PEAK_DATASHEET_TFLOPS} TFLOP/s)",
                         "flop64_per_launch": flop64, "kernel_ms": plain_s * 1e3,
                         "traffic": traffic, "traffic_source": traffic_src},
            "roofline_inference": {"bound": "tensor", "achieved": inf_flop / (inf_ms / 1e3) / 1e12,
                                   "peak": peak16, "unit": "TFLOP/s",
                                   "frac": inf_flop / (inf_ms / 1e3) / 1e12 / peak16,
                                   "peak_source": peak16_src, "flop_per_launch": inf_flop,
                                   "kernel_ms": inf_ms, "kernel": "surrogate inference (tcgen05), per step"},
            "cpu_baseline": cpu,
            "e2e": {"value": world * P * B / e2e_s, "unit": "pixel-bins/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3},
            "gpu_launches": 2 * args.steps,
            "clocks": clk,
            "secondary_c2": c2,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# Algorithmic BF16 work of one surrogate network on one (pixel, bin) sample:
# 64 -> 256, 3 x (256 -> 256), 256 -> 2 (multiply-add = 2 flop).
F_MLP = 2 * (64 * 256 + 3 * 256 * 256 + 256 * 2)


def measured_bf16_peak() -> tuple[float, str]:
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        if d.get("bf16_tflops"):
            return float(d["bf16_tflops"]), "MEASURED_PEAKS.json bf16_tflops (burst, cuBLAS 8192^3)"
    return 1590.0, "fallback 1.59 PFLOP/s (no MEASURED_PEAKS.json)"


def surrogate_arm(args) -> None:
    """Surrogate inference: the fused tcgen05 kernel evaluating an ensemble of
    4 networks on every (pixel, bin) of the config-4 inference image (mixed_512
    camera at 2048 x 2048, 32 bins).  Random weights: the kernel's work does not
    depend on their values."""
    import torch

    import hadros_b200 as hb
    from hadros_b200 import surrogate as S
    from hadros_b200 import workloads as W

    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    side, B, K = args.side or 2048, args.bins or 32, 4
    E, g2, sg = W.synthetic_sigma_arrays()
    sig = hb.SigmaTable.from_arrays(E, sg, g2)
    kw = W.surrogate_inference_image(nx=side, ny=side, n_bins=B)
    p = hb.params(**kw)
    P = side * side
    sur = S.Surrogate(members=K, device=local, seed=1)
    nm = hb.abi.HadrosMlpNorm()
    mu = [0.0, 0.0, 0.9, 0.5, 10.5] + [0.0] * 8 + [10.0, 0.3, 8.0]
    sd = [7.7, 7.7, 0.3, 0.3, 1.0] + [1.0] * 8 + [2.3, 0.1, 2.0]
    for j in range(16):
        nm.feat_mu[j], nm.feat_inv_sd[j] = mu[j], 1.0 / sd[j]
    nm.out_mu[0], nm.out_sd[0], nm.out_mu[1], nm.out_sd[1] = 5.0, 6.0, -60.0, 8.0
    nm.out_floor[0] = S.TAU_FLOOR
    sur.norm = nm
    out = S.alloc_image(P, B, device, per_bin=True)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)
    stream = torch.cuda.Stream(device=device)
    torch.cuda.set_stream(stream)
    for _ in range(args.warmup):
        sur.image(p, sig, threshold=0.005, out=out, stream=stream)
        flush.zero_()
    torch.cuda.synchronize()
    if out["counters"][1].item():
        raise RuntimeError("surrogate inference kernel aborted")
    gpu_index = local
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_index) as clocks:
        t_start.record(stream)
        for k in range(args.steps):
            ev[k][0].record(stream)
            sur.image(p, sig, threshold=0.005, out=out, stream=stream)
            ev[k][1].record(stream)
            flush.zero_()
        t_end.record(stream)
        torch.cuda.synchronize()
    clk = clocks.summary()
    per_step = max_over_ranks(t_start.elapsed_time(t_end) / 1e3) / args.steps
    kern_s = statistics.mean(a.elapsed_time(b) for a, b in ev) / 1e3
    achieved = P * B * K * F_MLP / kern_s / 1e12
    peak, peak_src = measured_bf16_peak()
    # e2e: the same call plus the per-pixel results read back to pinned host memory
    host = {k: torch.empty(out[k].shape, dtype=out[k].dtype, pin_memory=True)
            for k in ("tau", "P_surv", "I_obs", "spread")}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    d2h = 0
    for _ in range(args.steps):
        sur.image(p, sig, threshold=0.005, out=out, stream=stream, per_bin=False)
        for k, h in host.items():
            h.copy_(out[k], non_blocking=True)
        torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0) / args.steps
    d2h = sum(h.numel() * h.element_size() for h in host.values())
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        c = cpu_sample(kw, 160, host_threads())
        cpu = {"value": c["value"], "unit": "pixel-bins/s", "cores": c["cores"], "kind": c["kind"],
               "sample": describe_cpu(c, p.nx, p.ny) + " (the exact tracer the surrogate stands in for)"}
    if rank == 0:
        line = {
            "metric": "pixel-bins/sec", "value": world * P * B / per_step, "unit": "pixel-bins/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
            "data": "synthetic (random network weights; the work does not depend on them)",
            "config": {"workload": f"surrogate inference: ensemble of {K} networks (64 -> 4x256 -> 2) on "
                                   f"every pixel and bin of the mixed_512 camera at {side}x{side}, {B} bins",
                       "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"independent images, {world} GPU(s), no collective"},
            "samples_per_s": world * P * B * K / per_step,
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "peak_source": peak_src,
                         "flop_per_launch": P * B * K * F_MLP, "kernel_ms": kern_s * 1e3, "traffic": None},
            "cpu_baseline": cpu,
            "e2e": {"value": world * P * B / e2e_s, "unit": "pixel-bins/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3},
            "gpu_launches": args.steps,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["hadros", "reference", "reference-cuda"], default="hadros",
                    help="reference: the reference CPU code (the contract's reference arm); reference-cuda: "
                         "the reference's own GPU executable beside this library on one image")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["scan", "image", "surrogate"], default="scan",
                    help="scan: one production-scan point per step, surrogate + fallback + 1%% exact "
                         "judge (default); image: the trace kernel on mixed_512; surrogate: the "
                         "surrogate inference kernel alone")
    ap.add_argument("--epochs", type=int, default=150, help="scan: training epochs of the ensemble")
    ap.add_argument("--train-points", type=int, default=128, help="scan: training cameras (incl. held out)")
    ap.add_argument("--pixels-per-cam", type=int, default=4096, help="scan: training pixels per camera")
    ap.add_argument("--batch", type=int, default=8192, help="scan: training batch")
    ap.add_argument("--model", default=None,
                    help="scan: ensemble file (.npz): loaded when it exists (training record beside it), "
                         "else trained as usual and saved there")
    ap.add_argument("--lr", type=float, default=2e-3, help="scan: peak learning rate")
    ap.add_argument("--bound", type=float, default=0.01, help="scan: intensity error bound (fallback)")
    ap.add_argument("--judge", type=float, default=0.01, help="scan: judged fraction of pixels")
    ap.add_argument("--cpu-grid", type=int, default=64,
                    help="scan: CPU-baseline sample grid per side (64 x 64 = 4096 strided rays)")
    ap.add_argument("--ref-grid", type=int, default=REF_GRID,
                    help="scan, --impl reference: sample grid per side per step")
    ap.add_argument("--side", type=int, default=None, help="surrogate workload / reference-cuda: image side")
    ap.add_argument("--bins", type=int, default=None, help="surrogate workload: bins")
    ap.add_argument("--mev", action="store_true",
                    help="image workload: also run the MeV thermal channel (the reference arm's CPU "
                         "code always runs it)")
    args = ap.parse_args()
    if args.impl == "reference":
        if args.workload == "scan":
            reference_scan_arm(args)
        else:
            reference_arm(args)
    elif args.impl == "reference-cuda":
        reference_cuda_arm(args)
    elif args.workload == "surrogate":
        surrogate_arm(args)
    elif args.workload == "scan":
        scan_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
