"""The C ABI (include/hadros_b200.h) on the host: the library loads and
exports every declared function; parameters, names, sigma tables and error
behaviour follow the reference.  No GPU compute is called here."""
from __future__ import annotations

import ctypes as C
import math
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_functions() -> list[str]:
    text = (ROOT / "include" / "hadros_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hadros_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(hb):
    L = hb.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/hadros_b200.h but not exported"


def test_python_signatures_cover_header(hb):
    from hadros_b200 import abi
    assert set(declared_functions()) == set(abi.SIGNATURES)


def test_params_struct_size_and_defaults(hb):
    p = hb.params()
    assert p.struct_size == C.sizeof(hb.HadrosParams)
    assert p.tolerance == 1.0e-6 and p.max_steps == 200000
    assert p.h == 0.001 and p.fov_deg == 45.0 and p.nx == 100
    assert p.theta_obs_rad == math.pi * 74.0 / 180.0
    assert p.src_theta_width_rad == 8.0 * math.pi / 180.0
    assert p.spectral_kind == 0 and p.n_bins == 8
    assert hb.lib().hadros_params_validate(C.byref(p)) == 0


@pytest.mark.parametrize("alias,kind", [
    ("gaussian", 0), ("torus", 0), ("gaussian_torus", 0), ("powerlaw", 1), ("powerlaw_disk", 1),
    ("funnel", 2), ("gaussian_funnel", 2), ("powerlaw_funnel", 3), ("gaussian_envelope", 4),
    ("powerlaw_envelope", 5), ("powerlaw_funnel_envelope", 6), ("collapsar_ndaf_like", 7),
    ("collapsar_ndaf", 7)])
def test_profile_aliases(hb, alias, kind):
    assert hb.params(profile=alias).profile_kind == kind


@pytest.mark.parametrize("alias,kind", [
    ("inner_ring", 0), ("INNER_RING", 0), ("ring", 0), ("funnel_wall", 1), ("FUNNEL_WALL", 1),
    ("jet_base", 2), ("JET_BASE", 2), ("shock_layer", 3), ("SHOCK_LAYER", 3),
    ("density_weighted", 4), ("DENSITY_WEIGHTED", 4)])
def test_source_aliases(hb, alias, kind):
    assert hb.params(source=alias).source_kind == kind


@pytest.mark.parametrize("alias,kind", [
    ("monochromatic", 0), ("MONOCHROMATIC", 0), ("mono", 0), ("powerlaw", 1), ("POWERLAW", 1),
    ("power_law", 1), ("powerlaw_cutoff", 2), ("POWERLAW_CUTOFF", 2), ("power_law_cutoff", 2)])
def test_spectral_aliases(hb, alias, kind):
    assert hb.params(spectral=alias).spectral_kind == kind


def test_unknown_names_raise_reference_messages(hb):
    with pytest.raises(hb.HadrosError, match="Unknown density profile 'disk'"):
        hb.params(profile="disk")
    with pytest.raises(hb.HadrosError, match="Unknown UHE source model 'jet'"):
        hb.params(source="jet")
    with pytest.raises(hb.HadrosError, match="Unknown UHE spectral model 'flat'"):
        hb.params(spectral="flat")
    assert hb.lib().hadros_profile_name(6) == b"powerlaw_funnel_envelope"
    assert hb.lib().hadros_source_name(9) is None


@pytest.mark.parametrize("field,value", [("nx", 0), ("ny", -3), ("max_steps", 0),
                                         ("profile_kind", 8), ("source_kind", -1),
                                         ("spectral_kind", 3), ("precision", 2), ("h", 0.0),
                                         ("tolerance", -1.0), ("a_spin", float("nan"))])
def test_validate_rejects(hb, field, value):
    p = hb.params()
    setattr(p, field, value)
    assert hb.lib().hadros_params_validate(C.byref(p)) == 1
    assert hb.lib().hadros_last_error()


def test_validate_rejects_foreign_struct_size(hb):
    p = hb.params()
    p.struct_size = 12
    assert hb.lib().hadros_params_validate(C.byref(p)) == 1


def _write(tmp_path, rows, header=True):
    f = tmp_path / "s.dat"
    lines = ["# model test", "# Enu_GeV sigma_GeV_minus2 sigma_cm2"] if header else []
    f.write_text("\n".join(lines + rows) + "\n")
    return f


def test_sigma_file_parsing_follows_reference(hb, tmp_path):
    # comments, empty lines, unparsable and non-positive rows are skipped
    f = _write(tmp_path, ["1e4 1 2e-35", "", "# c", "garbage", "2e4 0 3e-35", "3e4 1 -1",
                          "5e4 2 4e-35", "1e5 3 5e-35"])
    t = hb.SigmaTable.load(f)
    assert t.info() == (3, 1.0e4, 1.0e5)
    assert t.sigma_cm2(1.0e4) == 2e-35
    assert t.sigma_cm2(1.0e5) == pytest.approx(5e-35, rel=1e-15)
    x = 7.0e4
    lx, l1, l2 = math.log(x), math.log(5e4), math.log(1e5)
    want = math.exp(math.log(4e-35) + (lx - l1) / (l2 - l1) * (math.log(5e-35) - math.log(4e-35)))
    assert t.sigma_cm2(x) == want


def test_sigma_errors(hb, tmp_path):
    with pytest.raises(hb.HadrosError, match="Could not open sigma table"):
        hb.SigmaTable.load(tmp_path / "missing.dat")
    with pytest.raises(hb.HadrosError, match="at least two valid data lines"):
        hb.SigmaTable.load(_write(tmp_path, ["1e4 1 2e-35"]))
    with pytest.raises(hb.HadrosError, match="strictly increasing"):
        hb.SigmaTable.load(_write(tmp_path, ["1e4 1 2e-35", "1e4 1 3e-35"]))
    t = hb.SigmaTable.load(_write(tmp_path, ["1e4 1 2e-35", "1e5 1 3e-35"]))
    with pytest.raises(hb.HadrosError) as e:
        t.sigma_cm2(1.0e6)
    assert e.value.status == 4 and "outside sigma table range" in e.value.message
    with pytest.raises(hb.HadrosError) as e:
        t.sigma_cm2(-1.0)
    assert e.value.status == 4


def test_sigma_eval_matches_oracle_on_synthetic(hb, sigma_table, sigma_arrays):
    E, _, s = sigma_arrays
    from oracle import pyoracle as O
    L = O.oracle_lib()
    for x in np.geomspace(E[0], E[-1], 97):
        assert sigma_table.sigma_cm2(float(x)) == L.hor_sigma_interp(
            E.ctypes.data, s.ctypes.data, int(E.size), float(x))


def test_spectral_bins_follow_reference_formula(hb, sigma_table):
    """integrate_kerr_ray_spectral's bins (src/radiative_transfer.cpp:711-737)."""
    p = hb.params(spectral="powerlaw_cutoff", n_bins=8, spec_e_min_GeV=1e5, spec_e_max_GeV=1e12,
                  spec_gamma=2.0, spec_ecut_GeV=1e12)
    b = hb.spectral_bins(p, sigma_table)
    e_min, e_max = max(1e5, 1e4), min(1e12, 1e12)
    lo, hi = math.log(e_min), math.log(e_max)
    d = (hi - lo) / 8.0
    for i in range(8):
        ll = lo + d * float(i)
        lr = ll + d
        em = math.exp(0.5 * (ll + lr))
        de = math.exp(lr) - math.exp(ll)
        w = max(em, 1e-300) ** -2.0 * math.exp(-max(em, 1e-300) / 1e12) * de
        assert b["E_mid"][i] == em and b["dE"][i] == de
        assert b["weight"][i] == pytest.approx(w, rel=1e-15)
        assert b["valid"][i] == 1
    empty = hb.spectral_bins(hb.params(spectral="powerlaw", spec_e_min_GeV=1e13,
                                       spec_e_max_GeV=1e14, n_bins=3), sigma_table)
    assert list(empty["valid"]) == [0, 0, 0]
    mono = hb.spectral_bins(hb.params(Enu_obs_GeV=3e7), sigma_table)
    assert list(mono["E_mid"]) == [3e7]


def test_null_handles_are_errors_not_crashes(hb, sigma_table):
    L = hb.lib()
    p = hb.params()
    out = hb.HadrosImageOut()
    assert L.hadros_image(None, C.byref(p), sigma_table.handle, C.byref(out)) == 7
    assert L.hadros_image_pixels(None, C.byref(p), sigma_table.handle, None, 0, C.byref(out)) == 1
    assert L.hadros_ctx_synchronize(None) == 7
    assert L.hadros_sigma_info(None, None, None, None) == 7
    L.hadros_ctx_destroy(None)
    L.hadros_sigma_destroy(None)


def test_context_without_gpu_reports_cuda_error(hb):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(hb.HadrosError) as e:
        hb.Context(0)
    assert e.value.status == 3


def test_ctypes_layouts_match_the_c_header(hb, tmp_path):
    """Every field of every struct in include/hadros_b200.h sits at the same
    offset (and every struct has the same size) in hadros_b200/abi.py: a C
    program compiled against the header prints them."""
    import shutil
    import subprocess
    from conftest import ROOT
    from hadros_b200 import abi
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"hadros_params": abi.HadrosParams, "hadros_image_out": abi.HadrosImageOut,
               "hadros_stats": abi.HadrosStats, "hadros_schedule": abi.HadrosSchedule,
               "hadros_mlp_norm": abi.HadrosMlpNorm, "hadros_adam": abi.HadrosAdam,
               "hadros_surrogate_out": abi.HadrosSurrogateOut, "hadros_train_sched": abi.HadrosTrainSched}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "hadros_b200.h"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'  printf("{name} sizeof %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(ROOT / "include"), "-o", str(exe), str(src)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        name, field, value = line.split()
        got[(name, field)] = int(value)
    for name, cls in structs.items():
        assert got[(name, "sizeof")] == C.sizeof(cls), name
        for field, _ in cls._fields_:
            assert got[(name, field)] == getattr(cls, field).offset, (name, field)

