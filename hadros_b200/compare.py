"""Image comparison: the aggregate metrics of the reference's CPU/CUDA
validation (scripts/compare_cuda_cpu_metrics.py:16-38: mean and max tau, mean
P_surv, total intensity over finite rows, uncaptured finite rays) and a
per-pixel comparison keyed by (i, j), independent of row order.

    python -m hadros_b200.compare REPORT.txt LABEL CPU.dat GPU.dat [LABEL CPU GPU ...]
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np


def load_image(path) -> np.ndarray:
    p = Path(path)
    if p.suffix == ".bin":
        import struct
        with open(p, "rb") as f:
            hdr = struct.Struct("<7i4d")
            magic, version, _backend, nx, ny, ncols, _r, *_ = hdr.unpack(f.read(hdr.size))
            if magic != 0x4B494D47 or version != 1:
                raise ValueError(f"not a KIMG v1 file: {path}")
            return np.fromfile(f, dtype="<f8").reshape(nx * ny, ncols)
    d = np.loadtxt(p, comments="#")
    return d.reshape(1, -1) if d.ndim == 1 else d


def metrics(d: np.ndarray) -> dict:
    tau, ps, inten, cap = d[:, 4], d[:, 5], d[:, 6], d[:, 7]
    finite = np.isfinite(tau) & np.isfinite(ps) & np.isfinite(inten)
    return {"mean_tau": float(np.mean(tau[finite])), "max_tau": float(np.max(tau[finite])),
            "mean_P_surv": float(np.mean(ps[finite])),
            "total_intensity": float(np.sum(inten[finite])),
            "valid_rays": int(np.count_nonzero(finite & (cap == 0)))}


def rel_diff(new, ref):
    if isinstance(ref, int):
        return new - ref
    if ref == 0.0:
        return 0.0 if new == 0.0 else float("inf")
    return (new - ref) / ref


def per_pixel(a: np.ndarray, b: np.ndarray) -> dict:
    """Max relative differences of tau and I matched by (i, j)."""
    ka = {(int(r[0]), int(r[1])): r for r in a}
    kb = {(int(r[0]), int(r[1])): r for r in b}
    common = sorted(set(ka) & set(kb))
    out = {"pixels": len(common), "captured_mismatch": 0, "max_rel_tau": 0.0, "max_rel_I": 0.0}
    for k in common:
        ra, rb = ka[k], kb[k]
        out["captured_mismatch"] += int(ra[7] != rb[7])
        for col, key in ((4, "max_rel_tau"), (6, "max_rel_I")):
            den = abs(ra[col])
            d = abs(rb[col] - ra[col]) / den if den > 0 else abs(rb[col] - ra[col])
            out[key] = max(out[key], d)
    return out


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) < 4 or (len(argv) - 1) % 3 != 0:
        print("Usage: python -m hadros_b200.compare REPORT.txt LABEL CPU.dat GPU.dat [...]")
        return 1
    lines = ["# CPU/GPU validation comparison", "# metric cpu gpu relative_difference",
             "# valid_rays reports gpu-cpu as an integer difference"]
    for i in range(1, len(argv), 3):
        label, cpu_path, gpu_path = argv[i], argv[i + 1], argv[i + 2]
        a, b = load_image(cpu_path), load_image(gpu_path)
        ma, mb = metrics(a), metrics(b)
        lines += ["", f"[{label}]", f"cpu_file {cpu_path}", f"gpu_file {gpu_path}"]
        for key in ("mean_tau", "max_tau", "mean_P_surv", "total_intensity", "valid_rays"):
            d = rel_diff(mb[key], ma[key])
            lines.append(f"{key} {ma[key]} {mb[key]} {d}" if key == "valid_rays"
                         else f"{key} {ma[key]:.16e} {mb[key]:.16e} {d:.16e}")
        pp = per_pixel(a, b)
        lines.append(f"per_pixel pixels={pp['pixels']} captured_mismatch={pp['captured_mismatch']} "
                     f"max_rel_tau={pp['max_rel_tau']:.3e} max_rel_I={pp['max_rel_I']:.3e}")
    Path(argv[0]).parent.mkdir(parents=True, exist_ok=True)
    Path(argv[0]).write_text("\n".join(lines) + "\n")
    print(argv[0])
    return 0


if __name__ == "__main__":
    sys.exit(main())
