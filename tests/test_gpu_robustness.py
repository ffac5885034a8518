"""The robustness scan (hadros_b200.robustness) on the GPU: all 47 cases in
one launch, against the same rows built from the CPU oracle.  Needs a B200."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_scan_in_one_launch_matches_oracle_rows(hb, gpu_ctx, sigma_table, sigma_arrays, tmp_path):
    from hadros_b200 import robustness as R
    from oracle import pyoracle as O
    E, _, s = sigma_arrays
    rows, stats = R.run(gpu_ctx, sigma_table, pixels=8, write_dat=str(tmp_path / "images"))
    assert len(rows) == 47 and stats["launches"] == 1 and stats["rays"] == 47 * 64
    table = R.cases()
    ref_rows = R.make_rows(table, [O.oracle_image(R.case_params(c, pixels=8)[0], E, s, mev=True) for c in table])
    for got, ref in zip(rows, ref_rows):
        assert (got["scan"], got["case"]) == (ref["scan"], ref["case"])
        assert got["valid_rays"] == ref["valid_rays"], got["case"]
        for k in ("mean_tau", "max_tau", "mean_P_surv", "total_intensity"):
            assert got[k] == pytest.approx(ref[k], rel=1e-6, abs=1e-300), (got["case"], k)
        assert got.get("anomaly", "") == ref.get("anomaly", "")
    # the .dat files carry the reference's names and the traced values
    f = rows[2]["output_file"]
    d = np.loadtxt(f, comments="#")
    assert d.shape == (64, 13)
    out = R.write_csv(rows, tmp_path)
    assert out.read_text().splitlines()[0].startswith("anomaly,aspin,cam_theta,case,")
    assert R.write_markdown(rows, tmp_path).read_text().startswith("# Robustness scan summary")


def test_spectral_validation_in_one_launch_matches_oracle(hb, gpu_ctx, sigma_table, sigma_arrays, tmp_path):
    from hadros_b200 import robustness as R
    from oracle import pyoracle as O
    E, _, s = sigma_arrays
    rows, stats = R.run_spectral(gpu_ctx, sigma_table, pixels=8)
    assert len(rows) == 6 and stats["launches"] == 1
    for (model, n, label), got in zip(R.spectral_cases(), rows):
        ref = R.spectral_metrics(O.oracle_image(R.spectral_params(model, n, pixels=8), E, s), label, n)
        assert got["valid_pixels"] == ref["valid_pixels"] and got["finite_outputs"] == ref["finite_outputs"]
        for k in ("mean_tau", "max_tau", "mean_Psurv", "integrated_intensity"):
            assert got[k] == pytest.approx(ref[k], rel=1e-6, abs=1e-300), (label, k)
    csv_path, md_path = R.write_spectral(rows, tmp_path)
    assert csv_path.read_text().splitlines()[0] == ("spectral_model,n_bins,mean_tau,max_tau,mean_Psurv,"
                                                    "integrated_intensity,valid_pixels,finite_outputs,"
                                                    "positive_weights")
    assert "powerlaw_cutoff convergence" in md_path.read_text()


def test_mev_bands_in_one_launch_match_oracle(hb, gpu_ctx, sigma_table, sigma_arrays, tmp_path):
    from hadros_b200 import robustness as R
    from test_robustness import _OracleContext
    E, _, s = sigma_arrays
    rows, grids, stats = R.run_mev_bands(gpu_ctx, sigma_table, pixels=8)
    assert len(rows) == 3 and stats["launches"] == 1
    ref_rows, ref_grids, _ = R.run_mev_bands(_OracleContext(E, s), None, pixels=8)
    for got, ref, g, rg in zip(rows, ref_rows, grids, ref_grids):
        assert got["integrated_I_mev"] == pytest.approx(ref["integrated_I_mev"], rel=1e-6), got["band"]
        np.testing.assert_allclose(g, rg, rtol=1e-6, atol=0.0)
    csv_path, ppm = R.write_mev_bands(rows, grids, tmp_path)
    assert ppm.read_bytes().startswith(b"P6\n8 8\n255\n")
