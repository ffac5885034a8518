"""bench.py's reference arm (CPU only): one JSON line with the contract's keys,
and ranks other than 0 print nothing."""
from __future__ import annotations

import json
import os
import subprocess
import sys

from conftest import ROOT


def _bench(*args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True, text=True,
                          timeout=600, env=e, cwd=ROOT)


def test_reference_arm_prints_one_contract_line():
    r = _bench("--impl", "reference", "--steps", "2", "--warmup", "1", "--ref-grid", "2")
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    c = d["cpu_baseline"]
    assert c["kind"] in ("reference", "port") and c["cores"] >= 1 and c["value"] == d["value"]
    assert c["value_mev_off"] > 0 and "workload" in d["config"]
    assert c["rays"] == 2 * 2 * 2 and c["steps_per_ray"] > 0


def test_reference_samples_are_disjoint_across_steps():
    sys.path.insert(0, str(ROOT))
    import bench
    seen = set()
    for k in range(20):
        ids = bench.ref_sample_ids(k)
        assert ids.size == bench.REF_GRID ** 2 and ids.min() >= 0 and ids.max() < bench.SCAN_SIDE ** 2
        assert seen.isdisjoint(ids.tolist())
        seen.update(ids.tolist())
    assert len(seen) >= 4096


def test_reference_arm_other_ranks_are_silent():
    r = _bench("--impl", "reference", "--steps", "1", "--warmup", "0", env={"RANK": "1"})
    assert r.returncode == 0 and r.stdout.strip() == ""
