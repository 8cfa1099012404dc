"""The reference's affine demo cases (examples/affine_bar_elastic.json, affine_shear_elastic.json)
through vpd.demo_runner on the GPU, against the reference CLI's output files
(tests/golden/example_outputs; the CLI built from the reference's sources, with the restated
elastic plugin, which this run loads too).

Run on CPU with the reference's own module functions, the same host code writes these files
byte for byte. On the GPU, F, the kinematics and the forces differ from the CPU by rounding.
So every column that carries a physical value must agree within 2e-5 of its largest entry:
the files print 6 digits. The rounding-noise columns (the F error, the net forces) must stay
below the case's own tolerances. Geometry and loading columns must agree as text."""
import csv
import gzip
import io
import json

import numpy as np
import pytest

from conftest import golden

import oracle as O
from vpd.demo_runner import run_demo_case

pytestmark = pytest.mark.gpu

NOISE = {"max_f_error": 1e-12, "net_force_x": 1e-7, "net_force_y": 1e-7, "net_force_z": 1e-7,
         "net_force_norm": 1e-7}
EXACT = {"material", "step", "time", "applied_strain", "elastic_reference_stress_xx",
         "elastic_reference_stress_xy", "finite", "particle", "x0", "y0", "z0", "ux", "uy", "uz",
         "x", "y", "z", "max_damage", "avg_damage", "damage", "internal_indicator",
         "avg_internal_indicator", "max_internal_indicator"}
F_COLUMNS = {"Fxx", "Fxy", "Fxz", "Fyx", "Fyy", "Fyz", "Fzx", "Fzy", "Fzz"}


def rows(text):
    r = list(csv.reader(io.StringIO(text)))
    return r[0], r[1:]


def compare(ours_text, ref_text):
    head, ours = rows(ours_text)
    ref_head, ref = rows(ref_text)
    assert head == ref_head and len(ours) == len(ref)
    for c, name in enumerate(head):
        if name in EXACT:
            assert [r[c] for r in ours] == [r[c] for r in ref], name
            continue
        a = np.array([float(r[c]) for r in ours])
        b = np.array([float(r[c]) for r in ref])
        if name in NOISE:
            assert np.abs(a).max() < NOISE[name] and np.abs(b).max() < NOISE[name], name
        elif name in F_COLUMNS:
            assert np.abs(a - b).max() <= 1e-12, name
        else:
            assert np.abs(a - b).max() <= 2e-5 * np.abs(b).max() + 1e-9, name


@pytest.mark.parametrize("case", ["affine_bar_elastic", "affine_shear_elastic"])
def test_affine_demo_matches_reference_cli(tmp_path, case):
    rc = run_demo_case(golden(f"examples/{case}.json"), str(tmp_path), golden(""), O.REF_DIR,
                       log=lambda *a: None)
    assert rc == 0

    def ref(name):
        with gzip.open(golden(f"example_outputs/{case}/{name}.gz"), "rt") as f:
            return f.read()

    compare((tmp_path / "timeseries.csv").read_text(), ref("timeseries.csv"))
    compare((tmp_path / "field_final.csv").read_text(), ref("field_final.csv"))
    meta = json.loads((tmp_path / "metadata.json").read_text())
    want = json.loads(ref("metadata.json"))
    for k in ("name", "status", "scope", "particles", "steps", "maxDamage", "allValuesFinite",
              "tolerances", "notes", "checks"):
        assert meta[k] == want[k], k
    assert meta["maxReferenceStressError"] == pytest.approx(want["maxReferenceStressError"], rel=1e-6)
    assert meta["maxDeformationGradientError"] < 1e-12 and meta["maxNetForceNorm"] < 1e-7
