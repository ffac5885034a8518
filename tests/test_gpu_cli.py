"""The command-line drop-in on the GPU: the reference executable's
--geodesic-cache and --image-from-cache modes give the in-line mode's image
(8x8 pixels, FP64).  Needs a B200."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CLI = ROOT / "hadros_b200" / "bin" / "compute_kerr_image"


def test_cache_modes_equal_the_in_line_image(tmp_path, sigma_arrays):
    from hadros_b200 import workloads as W
    E, g2, s = sigma_arrays
    for d in ("output/rays", "output/images", "data/sigma"):
        (tmp_path / d).mkdir(parents=True)
    W.write_sigma_file(tmp_path / "data" / "sigma" / "sigma_nuN_CC_GBW.dat", E, g2, s)
    run = lambda *a: subprocess.run([str(CLI), *a], cwd=tmp_path, capture_output=True, text=True,  # noqa: E731
                                    timeout=300)
    r = run("--geodesic-cache", "0.9", "60", "80", "25", "8", "8", "120", "0.05", "32", "50000", "1e-6")
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "output" / "rays" / "kerr_geodesics_cuda.bin").exists()
    physics = ["3", "1e10", "10", "5", "0.25", "3.5", "1", "15", "2", "1e12", "1", "10", "1", "80"]
    torus = ["gaussian", "2", "0", "15", "0", "2.5", "4", "60", "1e-3"]
    r = run("--image-from-cache", "1e9", "0.9", *physics, "256", *torus)
    assert r.returncode == 0, r.stderr
    r = run("1e9", "0.9", *physics, "60", "25", "8", "8", "120", "0.05", "32", "128", "200000", "1e-6", *torus,
            "--precision=fp64")
    assert r.returncode == 0, r.stderr
    dats = sorted((tmp_path / "output" / "images").glob("*.dat"))
    cached = [f for f in dats if "_cache_" in f.name]
    inline = [f for f in dats if "_cache_" not in f.name]
    assert len(cached) == 1 and len(inline) == 1
    assert cached[0].name.startswith("kerr_image_cuda_cache_rho0_torus_1e10_")
    a, b = np.loadtxt(cached[0]), np.loadtxt(inline[0])
    assert a.shape == b.shape == (64, 13)
    np.testing.assert_array_equal(a[:, 7], b[:, 7])           # captured
    np.testing.assert_array_equal(a[:, 4], b[:, 4])           # tau
    np.testing.assert_array_equal(a[:, 8:], b[:, 8:])         # the MeV columns
