"""Boundary-value case files through ``python -m vpd.runner`` on the GPU, against the
reference's own CLI (oracle/_ref/vumat_pd_run, built from its sources, run here on the CPU) on
the same file: a user plugin (the reference's linear elastic routine, restated in oracle/_ref)
through the host plugin path, and the device Johnson-Cook update from a configured initial
state.

Both write the same rows and keys. The numbers agree within 1e-7 of each column's scale,
because the GPU sums differ from the CPU's by rounding. The net internal force is rounding
noise in both, and it must stay under the case's 1e-6 N limit. The host plugin path matches
the reference library within 1e-9 in test_gpu_host_vumat.py."""
import csv
import io
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import golden

import oracle as O
from vpd.runner import run_boundary_case

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(
    not os.path.exists(os.path.join(O.REF_DIR, "vumat_pd_run")), reason="reference CLI not built")]
CLI = os.path.join(O.REF_DIR, "vumat_pd_run")


def pd_coarse_600(**material):
    with open(golden("cases/pd_coarse.json")) as f:
        case = json.load(f)
    dt = case["time_integration"]["dt"]
    case["time_integration"].update(steps=600, totalTime=600 * dt)
    case["materials"][0].update(material)
    case["output"] = {"directory": "out"}
    return case


def compare_with_reference_cli(tmp_path, case, plugin_dir=None):
    work = tmp_path / "ref"
    shutil.copytree(golden("configs"), work / "configs")
    (work / "cases").mkdir()
    path = work / "cases" / "case.json"
    path.write_text(json.dumps(case))
    ref = subprocess.run([CLI, "cases/case.json"], cwd=work, stdout=subprocess.DEVNULL)
    rc = run_boundary_case(str(path), str(tmp_path / "ours"), str(work), log=lambda *a: None,
                           plugin_dir=plugin_dir)
    assert rc == ref.returncode
    for name in ("timeseries.csv", "field_snapshots.csv"):
        a = list(csv.reader(io.StringIO((tmp_path / "ours" / name).read_text())))
        b = list(csv.reader(io.StringIO((work / "out" / name).read_text())))
        assert a[0] == b[0] and len(a) == len(b), name
        for c, col in enumerate(a[0]):
            if col in ("material", "step", "particle", "finite"):
                assert [r[c] for r in a[1:]] == [r[c] for r in b[1:]], (name, col)
                continue
            x = np.array([float(r[c]) for r in a[1:]])
            y = np.array([float(r[c]) for r in b[1:]])
            if col == "net_internal_force_N":
                assert np.abs(x).max() < 1e-6 and np.abs(y).max() < 1e-6
                continue
            assert np.abs(x - y).max() <= 1e-7 * np.abs(y).max() + 1e-12, (name, col)
    ours = json.loads((tmp_path / "ours" / "metadata.json").read_text())
    theirs = json.loads((work / "out" / "metadata.json").read_text())
    assert list(ours) == list(theirs)
    mo, mt = ours["materials"][0], theirs["materials"][0]
    assert list(mo) == list(mt) and mo["status"] == mt["status"]
    assert mo["finalReaction_N"] == pytest.approx(mt["finalReaction_N"], rel=1e-7)
    return mo, mt


def test_elastic_plugin_boundary_case_matches_reference_cli(tmp_path):
    mo, mt = compare_with_reference_cli(
        tmp_path, pd_coarse_600(materialConfigPath="configs/elastic.json", equivalentPlasticStrainIndex=-1),
        O.REF_DIR)
    assert mo["plugin_file"] == mt["plugin_file"] == "elastic_vumat_plugin.so"
    assert mo["maxEqps"] == mt["maxEqps"] == 0


def test_initial_state_boundary_case_matches_reference_cli(tmp_path):
    """JC from an initialised state with 1 % plastic strain already accumulated."""
    mo, mt = compare_with_reference_cli(tmp_path, pd_coarse_600(initialState=[1.0, 0.01, 293.0, 0.0, 0.0, 1.0]))
    assert mo["maxEqps"] == pytest.approx(mt["maxEqps"], rel=1e-7) and mt["maxEqps"] > 0.01


@pytest.mark.parametrize("indicator", [{"indices": [1], "reduction": "max"},
                                       {"indices": [1, 4], "reduction": "min", "transform": "one_minus"}])
def test_internal_indicator_boundary_case_matches_reference_cli(tmp_path, indicator):
    """The per-increment maximum of the indicator (k_indicator) and its per-point snapshot column."""
    mo, mt = compare_with_reference_cli(tmp_path, pd_coarse_600(internalIndicator=indicator))
    assert mo["maxInternalIndicator"] == pytest.approx(mt["maxInternalIndicator"], rel=1e-7)
    assert mt["maxInternalIndicator"] > 0
