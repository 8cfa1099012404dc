"""A boundary-value case file whose material is a user plugin (here the reference's linear
elastic routine, restated in oracle/_ref) through ``python -m vpd.runner --plugin-dir``: the
increments on the GPU around the host plugin path, against the reference's own CLI
(oracle/_ref/vumat_pd_run, built from its sources, run here on the CPU) on the same file.

Both write the same rows and keys. The numbers agree within 1e-7 of each column's scale,
because the GPU sums differ from the CPU's by rounding; the net internal force, rounding noise
in both, stays under the case's 1e-6 N limit. The host plugin path matches the
reference library within 1e-9 in test_gpu_host_vumat.py."""
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

pytestmark = [pytest.mark.gpu, pytest.mark.late]
CLI = os.path.join(O.REF_DIR, "vumat_pd_run")


@pytest.mark.skipif(not os.path.exists(CLI), reason="reference CLI not built")
def test_elastic_plugin_boundary_case_matches_reference_cli(tmp_path):
    with open(golden("cases/pd_coarse.json")) as f:
        case = json.load(f)
    dt = case["time_integration"]["dt"]
    case["time_integration"].update(steps=600, totalTime=600 * dt)
    case["materials"][0].update(materialConfigPath="configs/elastic.json", equivalentPlasticStrainIndex=-1)
    case["output"] = {"directory": "out"}
    work = tmp_path / "ref"
    shutil.copytree(golden("configs"), work / "configs")
    (work / "cases").mkdir()
    path = work / "cases" / "case.json"
    path.write_text(json.dumps(case))
    ref = subprocess.run([CLI, "cases/case.json"], cwd=work, stdout=subprocess.DEVNULL)
    rc = run_boundary_case(str(path), str(tmp_path / "ours"), str(work), log=lambda *a: None,
                           plugin_dir=O.REF_DIR)
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
            if col == "net_internal_force_N":  # rounding noise: under the case's 1e-6 N limit
                assert np.abs(x).max() < 1e-6 and np.abs(y).max() < 1e-6
                continue
            assert np.abs(x - y).max() <= 1e-7 * np.abs(y).max() + 1e-12, (name, col)
    ours = json.loads((tmp_path / "ours" / "metadata.json").read_text())
    theirs = json.loads((work / "out" / "metadata.json").read_text())
    assert list(ours) == list(theirs)
    mo, mt = ours["materials"][0], theirs["materials"][0]
    assert list(mo) == list(mt)
    assert mo["plugin_file"] == mt["plugin_file"] == "elastic_vumat_plugin.so"
    assert mo["status"] == mt["status"] and mo["maxEqps"] == mt["maxEqps"] == 0
    assert mo["finalReaction_N"] == pytest.approx(mt["finalReaction_N"], rel=1e-7)
