"""Shared fixtures.  Tests marked ``gpu`` need a B200 and the built CUDA
library; everything else runs on CPU."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 and libhadros_b200.so")


def golden_names(near_ties: bool = False) -> list[str]:
    """Fixture names; the scale_* fixtures (rays with near-tie accept/reject
    decisions, step counts held to +-1) only with near_ties=True."""
    names = sorted(p.stem for p in GOLDEN.glob("*.npz") if p.stem != "sigma_synthetic")
    return names if near_ties else [n for n in names if not n.startswith("scale_")]


def load_golden(name: str) -> tuple[dict, dict]:
    z = np.load(GOLDEN / f"{name}.npz")
    kw = json.loads(str(z["params"]))
    return kw, {k: z[k] for k in z.files if k != "params"}


@pytest.fixture(scope="session")
def sigma_arrays():
    z = np.load(GOLDEN / "sigma_synthetic.npz")
    return z["E"], z["sigma_GeV2"], z["sigma_cm2"]


@pytest.fixture(scope="session")
def hb():
    import hadros_b200
    hadros_b200.lib()
    return hadros_b200


@pytest.fixture(scope="session")
def sigma_table(hb, sigma_arrays):
    E, g2, s = sigma_arrays
    return hb.SigmaTable.from_arrays(E, s, g2)


@pytest.fixture(scope="session")
def gpu_ctx(hb):
    ctx = hb.Context(0)
    yield ctx
    ctx.close()
