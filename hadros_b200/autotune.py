"""Schedule autotuner for plans (hadros_plan_create).

The kernel's arithmetic is fixed; what a scan can still choose is its work
schedule: resident blocks per SM, the pixel order inside each camera (rows,
8x4 warp tiles, or descending cost from a coarse pre-pass) and whether costly
cameras are queued first.  The tuner times each candidate on a proxy of the
scan (every camera at 1/scale of its resolution per axis), keeps the fastest,
and caches the choice per GPU model and workload in a JSON file
($HADROS_B200_CACHE, default ~/.cache/hadros_b200/autotune.json).
"""
from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path

from . import ORDER_COST, ORDER_ROWS, ORDER_TILES, Context, SigmaTable, schedule

CANDIDATES = [dict(order=o, blocks_per_sm=b, camera_order=1)
              for o in (ORDER_ROWS, ORDER_TILES, ORDER_COST) for b in (0, 3)]


def _cache_file() -> Path:
    return Path(os.environ.get("HADROS_B200_CACHE", Path.home() / ".cache" / "hadros_b200" /
                               "autotune.json"))


def workload_key(cams: list, gpu_name: str) -> str:
    h = hashlib.sha256()
    for c in cams:
        h.update(bytes(c))
    return f"{gpu_name}:{h.hexdigest()[:16]}"


def proxy(cams: list, scale: int) -> list:
    out = []
    for c in cams:
        q = c.copy()
        q.nx = max(8, int(c.nx) // scale)
        q.ny = max(8, int(c.ny) // scale)
        out.append(q)
    return out


def autotune(ctx: Context, cams: list, sigma: SigmaTable, torch, scale: int = 4, repeats: int = 2,
             use_cache: bool = True) -> tuple:
    """Returns (best HadrosSchedule, report dict)."""
    gpu = torch.cuda.get_device_name(ctx.device)
    key = workload_key(cams, gpu)
    cf = _cache_file()
    cache = {}
    if use_cache and cf.exists():
        try:
            cache = json.loads(cf.read_text())
        except (OSError, ValueError):
            cache = {}
    if use_cache and key in cache:
        return schedule(**cache[key]["best"]), dict(cache[key], cached=True)
    px = proxy(cams, scale)
    stream = torch.cuda.current_stream()
    timings = []
    for cand in CANDIDATES:
        plan = ctx.plan(px, sigma, schedule(**cand))
        out = plan.alloc(torch, device=torch.device("cuda", ctx.device), outputs=("tau", "I_obs"))
        plan.launch(out, stream)            # warm-up
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(repeats):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.launch(out, stream)
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        timings.append({"schedule": cand, "ms": best})
        plan.close()
    win = min(timings, key=lambda t: t["ms"])
    report = {"best": win["schedule"], "timings": timings, "proxy_scale": scale, "gpu": gpu}
    if use_cache:
        cache[key] = report
        try:
            cf.parent.mkdir(parents=True, exist_ok=True)
            cf.write_text(json.dumps(cache, indent=1))
        except OSError:
            pass
    return schedule(**win["schedule"]), dict(report, cached=False)
