"""Every archived PD case file of the reference's tensile benchmark
(benchmarks/tensile3d/cases/pd_*.json) run on the GPU through the case-file runner, as
`vumat_pd_run CASE.json` runs it on the CPU:

  * the timeseries against the archived run's (raw/pd_*/timeseries.csv);
  * the final displacement at the analysis script's 1551 sample coordinates against the
    archived snapshot's;
  * the summary numbers of metadata.json against the archived ones;
  * the analysis metrics (vpd.metrics, the PD half of analyse_and_plot.py) against the frozen
    expected/analysis.json values with verify_metrics.py's 0.5 % tolerance.

Tolerances. The two 1,683-point cases hold the FP64 bar: stress history NRMSE below 1e-6,
the other columns, displacements and summaries within 1e-7 to 1e-8. The five 10,605-point
cases are chaotic at the last bit: the reference's own arithmetic with one component of the
deformation sum of every seventh point moved by one unit in the last place drifts from their
archive by several 1e-6 (tests/test_oracle.py::test_archived_shared_case_is_sensitive_to_one_ulp),
and the device sums the same bonds with other roundings (FMA, the stencil's slot order), so for
them the bar is the one such a rounding change meets: stress NRMSE below 3e-5, the reaction
within 1e-3 and the other quantities within 1e-4 of their peaks (measured on the device: 4e-6 to
1.1e-5 for the stress history, up to 2.6e-4 for the reaction; the reference's own run with the
one-ulp change: up to 7e-6 and 1e-4), and the analysis
metrics at verify_metrics.py's 0.5 % except final_stress_pct (see the test).
"""
import json
import math

import numpy as np
import pytest

from conftest import golden, max_rel, nrmse

from vpd import metrics as VM

pytestmark = pytest.mark.gpu

CASES = ("pd_coarse", "pd_delta2", "pd_delta4", "pd_dt12p5", "pd_dt50", "pd_m1p5", "pd_shared")


@pytest.fixture(scope="module")
def archive():
    data = np.load(golden("archived_pd_cases.npz"))
    with open(golden("expected_pd_metrics.json")) as f:
        expected = json.load(f)
    ref = {"stress": data["fem_reference_stress"], "u": data["fem_reference_u"],
           "final_stress": float(data["fem_reference_final_stress"]),
           "max_eqps": float(data["fem_reference_max_eqps"])}
    return data, expected, ref


CHAOTIC = {"pd_delta2", "pd_delta4", "pd_dt12p5", "pd_dt50", "pd_shared"}


@pytest.mark.parametrize("name", CASES)
def test_archived_case_runs_on_the_gpu(archive, name, tmp_path):
    from vpd.runner import run_boundary_case
    data, expected, ref = archive
    chaotic = name in CHAOTIC
    tol_stress, tol_col, tol_u, tol_sum = (3e-5, 1e-4, 1e-4, 1e-4) if chaotic else (1e-6, 1e-7, 1e-8, 1e-7)
    rc = run_boundary_case(golden(f"cases/{name}.json"), str(tmp_path), golden(""), log=lambda line: None)
    assert rc == 0  # the reference's acceptance verdict, as archived: pass
    mine = VM.read_csv(str(tmp_path / "timeseries.csv"))
    cols = [str(c) for c in data[f"{name}_columns"]]
    arch = {c: data[f"{name}_timeseries"][:, j] for j, c in enumerate(cols)}
    assert np.array_equal(mine["step"], arch["step"])
    assert nrmse(mine["average_axial_stress_MPa"], arch["average_axial_stress_MPa"]) < tol_stress
    for c in ("reaction_force_N", "max_eqps", "kinetic_energy_Nmm", "internal_energy_Nmm",
              "external_work_Nmm", "lateral_strain", "average_axial_strain", "load_displacement_mm"):
        # the reaction (a sum over the loaded band) is the noisiest column: the one-ulp change
        # moves it by up to 1e-4 of its peak in the reference's own arithmetic
        tol = 10 * tol_col if chaotic and c == "reaction_force_N" else tol_col
        assert max_rel(mine[c], arch[c]) < tol, c
    assert np.all(mine["finite"] == 1.0)

    snap = VM.read_csv(str(tmp_path / "field_snapshots.csv"))
    u = VM.interpolate_nodes(snap, VM.sample_coordinates())
    assert max_rel(u, data[f"{name}_u"]) < tol_u

    with open(tmp_path / "metadata.json") as f:
        meta = json.load(f)
    m = meta["materials"][0]
    max_eqps, reaction, energy_error, slope = data[f"{name}_summary"]
    assert meta["status"] == "pass" and m["status"] == "pass"
    assert m["maxEqps"] == pytest.approx(max_eqps, rel=tol_sum)
    assert m["finalReaction_N"] == pytest.approx(reaction, rel=10 * tol_sum if chaotic else tol_sum)
    assert m["finalEnergyError"] == pytest.approx(energy_error, rel=10 * tol_sum)
    assert m["earlyElasticSlope_MPa"] == pytest.approx(slope, rel=tol_sum)

    got = VM.run_metrics(str(tmp_path), ref)
    if not chaotic:
        assert VM.mismatches(expected[name], got) == [], (got, expected[name])
    else:
        # final_stress_pct is the difference of two nearly equal final stresses (0.06-0.2 %), so
        # a 1e-5 change of the final stress moves it by 1-2 %: the reference's own run with the
        # one-ulp change of the sensitivity test moves it by 1.4 % (pd_shared) and 1.9 %
        # (pd_delta2). It is checked through the final stress itself and in percentage points.
        assert VM.mismatches({k: v for k, v in expected[name].items() if k != "final_stress_pct"}, got) == []
        assert abs(got["final_stress_pct"] - expected[name]["final_stress_pct"]) < 0.01
        assert math.isclose(got["stress_MPa"], expected[name]["stress_MPa"], rel_tol=1e-4)
    for k in ("stress_history_pct", "displacement_pct", "max_eqps_pct"):
        assert math.isclose(got[k], expected[name][k], rel_tol=1e-2 if chaotic else 1e-5, abs_tol=1e-6), k
