"""The material-point case through the stock plugin, this package's library, so the
Johnson-Cook routine runs on the GPU (vumat_adapter_call of libvpd_gpu.so), against the
reference CLI's output files for examples/jc_material_point.json (tests/golden/example_outputs).

The GPU routine agrees with the restated Fortran routine to ~1e-12 per call; the plane-strain
bisection stops at a lateral stress below 1e-8 MPa, so the lateral strain may settle a few
1e-9 (relative) apart. Each numeric column must agree within 1e-6 of its largest value; the
step, time and load columns, which no plugin call touches, must agree exactly."""
import csv
import gzip
import io
import json

import numpy as np
import pytest

from conftest import golden

from vpd.point_runner import run_material_point_case

pytestmark = pytest.mark.gpu


def test_stock_jc_material_point_on_gpu(tmp_path):
    rc = run_material_point_case(golden("examples/jc_material_point.json"), str(tmp_path),
                                 config_root=golden(""), log=lambda *a: None)
    assert rc == 0
    with gzip.open(golden("example_outputs/jc_material_point/timeseries.csv.gz"), "rt") as f:
        ref = list(csv.reader(io.StringIO(f.read())))
    ours = list(csv.reader(io.StringIO((tmp_path / "timeseries.csv").read_text())))
    assert ours[0] == ref[0] and len(ours) == len(ref) == 601
    col = {k: i for i, k in enumerate(ref[0])}
    for k in ("material", "step", "time", "applied_strain", "elastic_reference_stress", "finite"):
        assert [r[col[k]] for r in ours[1:]] == [r[col[k]] for r in ref[1:]], k
    for k in ("stress", "reference_error", "state_indicator", "internal_energy", "inelastic_energy",
              "temperature", "lateral_strain"):
        a = np.array([float(r[col[k]]) for r in ours[1:]])
        b = np.array([float(r[col[k]]) for r in ref[1:]])
        assert np.max(np.abs(a - b)) <= 1e-6 * np.max(np.abs(b)), k
    meta = json.loads((tmp_path / "metadata.json").read_text())
    with gzip.open(golden("example_outputs/jc_material_point/metadata.json.gz"), "rt") as f:
        ref_meta = json.load(f)
    assert meta["status"] == ref_meta["status"] == "pass"
    m, r = meta["materials"][0], ref_meta["materials"][0]
    for k in ("finalStress", "finalIndicator", "finalInternalEnergy", "finalInelasticEnergy"):
        assert m[k] == pytest.approx(r[k], rel=1e-7), k
