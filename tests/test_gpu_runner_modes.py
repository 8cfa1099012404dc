"""The archived pd_coarse case file on the headline path: ``python -m vpd.runner
--precision mixed --surrogate hybrid`` (FP32 bond sums, the learned Johnson-Cook return map
trained on the GPU first, the VUMAT as fallback), against the reference's archived run of the
same file at the stated tolerance for these forms (stress-history NRMSE <= 0.5 %).

The case's acceptance limits hold except the net internal force's. That limit is 1e-6 N, a
bound on FP64 round-off, and FP32 bond sums exceed it by construction. So the runner reports
the reference's verdict, ``fail``, and the test checks each of the other limits itself, and
that the net force stays small next to the reaction."""
import csv
import gzip
import io
import json

import numpy as np
import pytest

from conftest import golden, nrmse

from vpd.runner import main

pytestmark = pytest.mark.gpu


def test_case_file_on_the_surrogate_mixed_path(tmp_path):
    rc = main([golden("cases/pd_coarse.json"), "--config-root", golden(""), "--out", str(tmp_path),
               "--precision", "mixed", "--surrogate", "hybrid"])
    assert rc in (0, 2)
    meta = json.loads((tmp_path / "metadata.json").read_text())
    m, acc = meta["materials"][0], meta["acceptance"]
    assert m["finite"] and m["finalEnergyError"] <= acc["energyToleranceRelative"]
    assert m["finalKineticToInternal"] <= acc["kineticToInternalLimit"]
    assert m["maxEqps"] >= acc["minimumPlasticStrain"]
    assert m["maxEqps"] == pytest.approx(0.0278018224371612, rel=1e-3)  # the archived run's
    assert m["maxNetInternalForce_N"] < 1e-3 * abs(m["finalReaction_N"])
    ours = list(csv.reader(io.StringIO((tmp_path / "timeseries.csv").read_text())))
    with gzip.open(golden("pd_coarse_timeseries.csv.gz"), "rt") as f:
        ref = list(csv.reader(f))
    assert ours[0] == ref[0] and len(ours) == len(ref)
    col = ref[0].index("average_axial_stress_MPa")
    a = np.array([float(r[col]) for r in ours[1:]])
    b = np.array([float(r[col]) for r in ref[1:]])
    assert nrmse(a, b) <= 5e-3
