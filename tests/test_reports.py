"""Run reports in the reference driver's layout (CPU).

error_stats must be the statistics of utils/utils.cpp:60-125, and a log made
by format_run_log must be read by the reference's own
utils/parse_glst_results.py into the fields its CSV has (run only where the
environment variable REF_ROOT names the reference source tree; the script is
imported, not copied).
"""
import importlib.util
import math
import os
import types

import numpy as np
import pytest

REF_PARSER = os.path.join(os.environ.get("REF_ROOT", ""), "utils", "parse_glst_results.py")


def _info():
    return types.SimpleNamespace(natom=30000, ncell=(7, 7, 7), cell_dim=10.0, ngroup=3, num_nodes=100532,
                                 group_nodes=[60522, 30510, 9500] + [0] * 13)


def _stats(pkg, seed=0, n=500):
    from glst_b200 import reports
    rng = np.random.default_rng(seed)
    glst = [rng.normal(size=n) for _ in range(4)]
    coul = [g + 1e-6 * rng.normal(size=n) for g in glst]
    return reports.error_stats(glst, coul), glst, coul


def test_error_stats_follow_the_reference_definitions(pkg):
    st, glst, coul = _stats(pkg)
    for i, comp in enumerate(("fx", "fy", "fz", "en")):
        err = coul[i] - glst[i]
        rms_g = math.sqrt(np.mean(glst[i] ** 2))
        assert st[comp]["min"][0] == np.abs(err).min()
        assert st[comp]["max"][0] == np.abs(err).max()
        assert math.isclose(st[comp]["avg"][0], np.abs(err).mean(), rel_tol=1e-12)
        assert math.isclose(st[comp]["rms"][0], math.sqrt(np.mean(err ** 2)), rel_tol=1e-12)
        assert math.isclose(st[comp]["rms"][1], st[comp]["rms"][0] / rms_g, rel_tol=1e-12)


def _log(pkg):
    from glst_b200 import reports
    st, _, _ = _stats(pkg)
    meta = {"sweep": "bench", "sys": "water10k", "tol": "1.16487e-06", "box_dim": "66.9,66.9,66.9", "cut": "10",
            "requested_gpus": "1"}
    per = {"assign": [0.03, 0.04], "near_field": [0.29, 0.31], "structure_factors": [1.28, 1.30],
           "shell_sums": [0.44, 0.46], "long_range": [1.56, 1.58], "combine": [0.04, 0.04]}
    return reports.format_run_log(meta, _info(), (66.9, 66.9, 66.9), per, 12.5, st, 1.16487e-06), st


def test_log_layout(pkg):
    text, _ = _log(pkg)
    assert text.startswith("BENCH_INPUT sweep=bench sys=water10k tol=1.16487e-06")
    assert "          Number of cells: 7, 7, 7" in text
    assert "  Number of cubature nodes in group 2: 9500" in text
    assert "             Calculate structure factors: 1.29 ms (+/- 0.01 ms)" in text
    assert "Finished 2 calculations" in text


def test_reference_parser_reads_the_log(pkg, tmp_path):
    if not os.path.exists(REF_PARSER):
        pytest.skip("reference sources not present")
    spec = importlib.util.spec_from_file_location("parse_glst_results", REF_PARSER)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    text, st = _log(pkg)
    path = tmp_path / "run.log"
    path.write_text(text)
    row = mod.parse_file(path)
    assert row["sys"] == "water10k" and row["cut"] == "10" and row["requested_gpus"] == "1"
    assert row["num_atoms"] == 30000 and row["num_gpus"] == 1 and row["alpha_groups"] == 3
    assert row["cubature_nodes_total"] == 100532
    assert row["cubature_nodes_by_group"] == "60522|30510|9500"
    assert (row["ncell_x"], row["ncell_y"], row["ncell_z"]) == ("7", "7", "7")
    assert row["iterations"] == 2
    assert math.isclose(row["calc_sf_ms"], 1.29) and math.isclose(row["calc_sf_std_ms"], 0.01)
    assert math.isclose(row["total_ms"], 0.035 + 0.30 + 1.29 + 0.45 + 1.57 + 0.04)
    assert math.isclose(row["coulomb_ms"], 12.5)
    assert math.isclose(row["err_fx_rms"], st["fx"]["rms"][0], rel_tol=1e-6)
    assert math.isclose(row["norm_en_max"], st["en"]["max"][1], rel_tol=1e-6)


def _golden_logs():
    here = os.path.join(os.path.dirname(__file__), "golden")
    return {k: os.path.join(here, v) for k, v in (("ref", "full_example_water10k_ref.log"),
                                                   ("b200", "full_example_water10k_b200.log"),
                                                   ("bench", "bench_water10k.log"))}


def test_recorded_driver_logs_side_by_side(tmp_path):
    """Logs recorded on a B200 by oracle/run_drivers.py (the reference's
    driver against the reference library and, unchanged, against this engine)
    and by bench.py --reference-log, read by the reference's parser: same
    system, grid and node counts; the RMS error against direct Coulomb of the
    forces within 1 % of the reference library's, of the per-atom energies
    within 6 % (FP32 phases: per-atom energies carry ~1e-6 relative rounding,
    the total energy 1e-9)."""
    if not os.path.exists(REF_PARSER):
        pytest.skip("reference sources not present")
    spec = importlib.util.spec_from_file_location("parse_glst_results", REF_PARSER)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    from pathlib import Path
    rows = {k: mod.parse_file(Path(p)) for k, p in _golden_logs().items()}
    same = ("num_atoms", "ncell_x", "ncell_y", "ncell_z", "alpha_groups", "cubature_nodes_total",
            "cubature_nodes_by_group", "cell_x", "system_x")
    for k in ("b200", "bench"):
        for f in same:
            assert rows[k][f] == rows["ref"][f], (k, f)
        for comp, rel in (("fx", 0.01), ("fy", 0.01), ("fz", 0.01), ("en", 0.06)):
            assert math.isclose(rows[k]["err_%s_rms" % comp], rows["ref"]["err_%s_rms" % comp], rel_tol=rel)
    assert rows["b200"]["total_ms"] < rows["ref"]["total_ms"] / 5
