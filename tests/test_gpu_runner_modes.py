"""The archived pd_coarse case file on the headline path: ``python -m vpd.runner
--precision mixed --surrogate hybrid`` (FP32 bond sums, the learned Johnson-Cook return map
trained on the GPU first, the VUMAT as fallback), against the reference's archived run of the
same file at the stated tolerance for these forms (stress-history NRMSE <= 0.5 %)."""
import csv
import gzip
import io

import numpy as np
import pytest

from conftest import golden, nrmse

from vpd.runner import main

pytestmark = [pytest.mark.gpu, pytest.mark.late]


def test_case_file_on_the_surrogate_mixed_path(tmp_path):
    rc = main([golden("cases/pd_coarse.json"), "--config-root", golden(""), "--out", str(tmp_path),
               "--precision", "mixed", "--surrogate", "hybrid"])
    assert rc == 0  # the archived run passes its acceptance limits; so must this one
    ours = list(csv.reader(io.StringIO((tmp_path / "timeseries.csv").read_text())))
    with gzip.open(golden("pd_coarse_timeseries.csv.gz"), "rt") as f:
        ref = list(csv.reader(f))
    assert ours[0] == ref[0] and len(ours) == len(ref)
    col = ref[0].index("average_axial_stress_MPa")
    a = np.array([float(r[col]) for r in ours[1:]])
    b = np.array([float(r[col]) for r in ref[1:]])
    assert nrmse(a, b) <= 5e-3
