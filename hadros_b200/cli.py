"""Command-line entry: trace a named workload image through the C ABI.

    python -m hadros_b200.cli image --workload mixed_512 [--nx 256 --ny 256]
           [--precision mixed|fp64] [--repeat N] [--sigma FILE] [--mev]

Prints one JSON line with the run statistics (rays, accepted steps, attempts,
kernel time, fates).  --mev also runs the MeV thermal channel.  The
reference's own command-line drop-in (compute_kerr_image, positional argv) is
the executable hadros_b200/bin/compute_kerr_image.
"""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np

from . import Context, SigmaTable, params
from . import workloads as W

WORKLOADS = {"plain_tracer_32": W.plain_tracer_32, "mixed_512": W.mixed_512,
             "production_point": W.production_point}


def cmd_image(a) -> int:
    kw = WORKLOADS[a.workload]()
    for k in ("nx", "ny", "precision", "n_bins", "max_steps"):
        v = getattr(a, k)
        if v is not None:
            kw[k] = v
    if a.mev:
        kw["mev_channel"] = 1
    p = params(**kw)
    if a.sigma:
        sig = SigmaTable.load(a.sigma)
    else:
        E, g2, s = W.synthetic_sigma_arrays()
        sig = SigmaTable.from_arrays(E, s, g2)
    with Context(a.device) as ctx:
        ctx.set_transfer(a.transfer)
        for r in range(a.repeat):
            img = ctx.image(p, sig, outputs=("tau", "I_obs", "fate", "steps", "attempts"))
            st = ctx.stats()
            fates = np.bincount(img["fate"].astype(np.int64), minlength=3)
            print(json.dumps({"workload": a.workload, "nx": p.nx, "ny": p.ny, "bins": int(p.n_bins),
                              "transfer": a.transfer, "mev_channel": int(p.mev_channel),
                              "precision": int(p.precision), "repeat": r,
                              "kernel_ms": st["kernel_ms"], "total_ms": st["total_ms"],
                              "rays": st["rays"], "accepted_steps": st["accepted_steps"],
                              "attempts": st["attempts"],
                              "fates": {"escaped": int(fates[0]), "captured": int(fates[1]),
                                        "truncated": int(fates[2])},
                              "sum_I": float(img["I_obs"].sum()),
                              "mean_tau": float(img["tau"].mean())}), flush=True)
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m hadros_b200.cli", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    im = sub.add_parser("image", help="trace a workload image")
    im.add_argument("--workload", choices=sorted(WORKLOADS), default="mixed_512")
    im.add_argument("--nx", type=int)
    im.add_argument("--ny", type=int)
    im.add_argument("--n-bins", dest="n_bins", type=int)
    im.add_argument("--max-steps", dest="max_steps", type=int)
    im.add_argument("--precision", choices=["fp64", "mixed"])
    im.add_argument("--repeat", type=int, default=1)
    im.add_argument("--transfer", choices=["auto", "in_loop", "deferred"], default="auto",
                    help="mixed precision: per-point transfer in the loop, or deferred (warp replays)")
    im.add_argument("--device", type=int, default=0)
    im.add_argument("--sigma", help="sigma table file (reference 3-column format)")
    im.add_argument("--mev", action="store_true", help="also run the MeV thermal channel")
    a = ap.parse_args(argv)
    if a.cmd == "image":
        return cmd_image(a)
    return 2


if __name__ == "__main__":
    sys.exit(main())
