"""The case-file runner's host side, on CPU: the reference's case files read into cases, and
the output writers checked against the reference's archived output text.

The writers are pinned by feeding them the archived run's own values
(benchmarks/tensile3d/raw/pd_coarse, fixtures in tests/golden) and comparing the text byte for
byte; running a case on the GPU is covered in test_gpu_parity.py."""
import csv
import gzip
import json
import math
import os

import numpy as np
import pytest

from conftest import golden

from vpd.boundary_case import load_boundary_case
from vpd.case import DIAG, DIAG_COLUMNS, pd_coarse
from vpd.runner import (SNAPSHOT_HEADER, TIMESERIES_HEADER, metadata_text, observation_bounds,
                        snapshot_lines, snapshot_steps, summarise, timeseries_line)

CASES = sorted(f for f in os.listdir(golden("cases")) if f.endswith(".json"))


def case_path(name):
    return os.path.join(golden("cases"), name)


def load(name):
    return load_boundary_case(case_path(name), golden(""))


@pytest.mark.parametrize("name", CASES)
def test_archived_case_files_load(name):
    bc = load(name)
    c = bc.materials[0].case
    assert c.n_points > 0 and c.horizon > c.spacing and bc.steps * c.dt == pytest.approx(0.12)
    assert bc.materials[0].label == "JC" and bc.materials[0].eqps_index == 1
    assert os.path.basename(name)[:-5] == bc.name


def test_pd_coarse_file_is_the_hand_written_case():
    c = load("pd_coarse.json").materials[0].case
    ref = pd_coarse()
    for field in ("nx", "ny", "nz", "spacing", "horizon", "dt", "steps", "density", "props",
                  "bc_mode", "load_axis", "region_layers", "plane_strain", "amplitude", "rise_time",
                  "observation_min", "observation_max", "nstatev", "reference_temperature",
                  "damage_mode"):
        assert getattr(c, field) == getattr(ref, field), field


@pytest.mark.parametrize("edit, message", [
    (lambda d: d["boundary_conditions"].update(type="affine_displacement"), "regional_smooth_displacement"),
    (lambda d: d["boundary_conditions"].update(supportRegion="right", loadRegion="left"), "support"),
    (lambda d: d["boundary_conditions"].update(rigidBodySuppression=False), "rigidBodySuppression"),
    (lambda d: d["boundary_conditions"].update(component="z"), "component"),
    (lambda d: d["damage"].update(model="bond_based"), "damage.model"),
    (lambda d: d.update(type="vumat_material_point_case"), "vumat_pd_boundary_case"),
    (lambda d: d["materials"][0].update(internalIndicator={"indices": [1], "reduction": "sum"}), "reduction must be"),
    (lambda d: d["materials"][0].update(internalIndicator={"indices": [6]}), "outside nstatev"),
    (lambda d: d["materials"][0].update(initialStateOverrides={"1x": 0.1}), "initialStateOverrides index"),
    (lambda d: d["materials"][0].update(initialState=[0.0, 0.1]), "initialState length"),
    (lambda d: d["materials"][0].update(materialConfigPath="configs/elastic.json"), "elastic.json"),
])
def test_unsupported_case_files_are_refused(tmp_path, edit, message):
    with open(case_path("pd_coarse.json")) as f:
        d = json.load(f)
    edit(d)
    p = tmp_path / "case.json"
    p.write_text(json.dumps(d))
    with pytest.raises((ValueError, OSError)) as e:
        load_boundary_case(str(p), golden(""))
    assert message in str(e.value)


def test_point_damage_modes_load(tmp_path):
    """The point modes and deletionEnabled pass through; failure defaults to 1 as in
    SimpleDamageConfig (include/SimpleDamageModel.hpp:13-15)."""
    with open(case_path("pd_coarse.json")) as f:
        d = json.load(f)
    d["damage"] = {"model": "eqps_threshold", "initiation": 0.002, "deletionEnabled": True}
    p = tmp_path / "case.json"
    p.write_text(json.dumps(d))
    c = load_boundary_case(str(p), golden("")).materials[0].case
    assert (c.damage_mode, c.damage_initiation, c.damage_failure, c.damage_deletion) == (2, 0.002, 1.0, True)
    d["damage"] = {"model": "max_principal_strain", "initiation": 0.005, "failure": 0.03}
    p.write_text(json.dumps(d))
    c = load_boundary_case(str(p), golden("")).materials[0].case
    assert (c.damage_mode, c.damage_failure, c.damage_deletion) == (3, 0.03, False)


def archived_timeseries():
    with gzip.open(golden("pd_coarse_timeseries.csv.gz"), "rt") as f:
        text = f.read()
    rows = list(csv.reader(text.splitlines()))
    return text, rows[0], rows[1:]


def test_timeseries_writer_reproduces_archived_text():
    text, header, body = archived_timeseries()
    assert TIMESERIES_HEADER == ",".join(header) + "\n"
    out = [TIMESERIES_HEADER]
    for r in body:
        row = np.zeros(len(DIAG_COLUMNS))
        for name, value in zip(header[1:], r[1:]):
            row[DIAG[name if name != "finite" else "finite"]] = float(value)
        out.append(timeseries_line(r[0], row))
    assert "".join(out) == text


def test_snapshot_writer_reproduces_archived_text():
    with gzip.open(golden("pd_coarse_snapshot_head.csv.gz"), "rt") as f:
        text = f.read()
    rows = list(csv.reader(text.splitlines()))
    header, body = rows[0], rows[1:]
    assert SNAPSHOT_HEADER == ",".join(header) + "\n"
    col = {k: i for i, k in enumerate(header)}

    def arr(*names):
        return np.array([[float(r[col[k]]) for k in names] for r in body])

    x0 = arr("x0_mm", "y0_mm", "z0_mm")
    u = arr("ux_mm", "uy_mm", "uz_mm")
    v = arr("vx_mm_per_ms", "vy_mm_per_ms", "vz_mm_per_ms")
    lines = snapshot_lines("JC", 4800, 0.12, x0, u, v, arr("axial_strain")[:, 0],
                           arr("axial_stress_MPa")[:, 0], arr("eqps")[:, 0], arr("simple_damage")[:, 0])
    got = list(csv.reader(lines.splitlines()))
    assert len(got) == len(body)
    current = {"x_mm", "y_mm", "z_mm"}  # x0 + u: recomputed from the printed x0 and u
    for g, r in zip(got, body):
        assert [a for k, a in zip(header, g) if k not in current] == \
               [a for k, a in zip(header, r) if k not in current]
        for k in current:
            assert float(g[col[k]]) == pytest.approx(float(r[col[k]]), rel=1e-15, abs=1e-15)


def test_summary_of_the_archived_run():
    """The summary fields that the archived output rows determine (the final increment and the
    monotone max eqps) agree with the archived metadata at its 15 digits."""
    _, header, body = archived_timeseries()
    rows = np.zeros((len(body), len(DIAG_COLUMNS)))
    for k, name in enumerate(header[1:]):
        rows[:, DIAG[name]] = [float(r[k + 1]) for r in body]
    s = summarise(rows, 210000.0, 0.3)
    meta = {"maxEqps": 0.0278018224371612, "finalReaction": 9875.54163611348,
            "finalNominalStress": 123.444270451419, "finalEngineeringStrain": 0.0204081632653061,
            "finalEnergyError": 0.0224015614675876, "analyticalPlaneStrainSlope": 230769.230769231}
    for k, v in meta.items():
        assert "%.15g" % s[k] == "%.15g" % v, k
    assert s["finite"]


def test_metadata_is_json_in_the_reference_layout():
    bc = load("pd_coarse.json")
    s = {"pass": True, "runtimeSeconds": 1.25, "observationMin": 2.0, "observationMax": 98.0,
         "maxNetInternalForce": 3.3e-10, "finalEnergyError": 0.0224, "maxEnergyError": 0.0224,
         "maxKineticToInternal": 2424.5, "finalKineticToInternal": 0.0023, "maxEqps": 0.0278,
         "maxInternalIndicator": 0.0, "earlyElasticSlope": 201234.9, "analyticalPlaneStrainSlope": 230769.2,
         "earlyElasticRelativeError": 0.128, "finalReaction": 9875.5, "finalNominalStress": 123.4,
         "finalEngineeringStrain": 0.0204, "finite": True}
    text = metadata_text(bc, [s])
    d = json.loads(text)
    assert list(d) == ["name", "solver", "status", "classification", "scope", "units",
                       "densityConversion", "particles", "grid", "spacing_mm", "horizon_mm",
                       "horizonSpacingRatio", "neighborSearch", "planeStrain", "outerSimpleDamage",
                       "zeroEnergyStabilization", "timeStepPolicy", "boundarySets", "dt_ms", "steps",
                       "materials", "acceptance", "materialComparisonCaveat", "parameterMatchingPolicy",
                       "legacyBlockPolicy"]
    assert d["particles"] == 1683 and d["grid"] == [51, 11, 3] and d["status"] == "pass"
    assert '"dt_ms": 2.5e-05,' in text  # the stream's default 6 digits, as the archive has it
    m = d["materials"][0]
    assert m["name"] == "JC" and m["observationAxis"] == "x" and m["sourceDensity_kg_per_m3"] == 7800
    assert d["acceptance"] == {"energyToleranceRelative": 0.15, "netForceTolerance_N": 1e-06,
                               "minimumPlasticStrain": 0.001, "kineticToInternalLimit": 10}
    s["finalEnergyError"] = math.inf
    assert '"finalEnergyError": null' in metadata_text(bc, [s])


def test_snapshot_steps_and_observation_window():
    bc = load("pd_coarse.json")
    assert snapshot_steps(bc) == [4800]
    bc.snapshot_every = 1000
    assert snapshot_steps(bc) == [1000, 2000, 3000, 4000, 4800]
    bc.snapshot_every = 0
    assert snapshot_steps(bc) == [4800]
    x = np.stack(np.meshgrid(np.arange(51) * 2.0, np.arange(11) * 2.0 - 10, [-2.0, 0.0, 2.0],
                             indexing="ij"), -1).reshape(-1, 3)
    assert observation_bounds(x, 0, 2.0, math.nan, math.nan) == (2.0, 98.0)
    assert observation_bounds(x, 0, 2.0, 10.0, 90.0) == (10.0, 90.0)
    with pytest.raises(ValueError):
        observation_bounds(x, 0, 2.0, 50.0, 40.0)


def test_boundary_case_with_a_host_plugin(tmp_path):
    """A material config naming another plugin loads for the host plugin path: its props,
    state count and plugin are kept for set_host_vumat, the case carries the device layout's
    6 state columns, and eqps must be state variable 2 or none."""
    import oracle as O
    with open(case_path("pd_coarse.json")) as f:
        d = json.load(f)
    d["materials"][0].update(materialConfigPath="configs/elastic.json", equivalentPlasticStrainIndex=-1)
    p = tmp_path / "case.json"
    p.write_text(json.dumps(d))
    m = load_boundary_case(str(p), golden(""), O.REF_DIR).materials[0]
    assert m.host_plugin is not None and m.host_plugin.nstatev == 1 and m.host_plugin.props == (210000.0, 0.3)
    assert os.path.basename(m.host_plugin.plugin_path) == "elastic_vumat_plugin.so"
    assert m.case.nstatev == 6 and m.case.props == (0.0,) * 14 and m.eqps_index == -1
    d["materials"][0]["equivalentPlasticStrainIndex"] = 0
    p.write_text(json.dumps(d))
    with pytest.raises(ValueError, match="must be 1 or -1"):
        load_boundary_case(str(p), golden(""), O.REF_DIR)
    assert load_boundary_case(case_path("pd_coarse.json"), golden("")).materials[0].host_plugin is None


def test_runner_surrogate_option_checks(tmp_path):
    """The surrogate replaces the device JC update only, and takes the library's guess names;
    both are refused before any GPU work."""
    import oracle as O
    from vpd.runner import main, run_boundary_case
    with open(case_path("pd_coarse.json")) as f:
        d = json.load(f)
    d["materials"][0].update(materialConfigPath="configs/elastic.json", equivalentPlasticStrainIndex=-1)
    p = tmp_path / "case.json"
    p.write_text(json.dumps(d))
    with pytest.raises(ValueError, match="not a host plugin"):
        run_boundary_case(str(p), str(tmp_path / "o"), golden(""), plugin_dir=O.REF_DIR, surrogate="hybrid")
    with pytest.raises(ValueError, match="one of"):
        run_boundary_case(case_path("pd_coarse.json"), str(tmp_path / "o"), golden(""), surrogate="fast")
    with pytest.raises(SystemExit):
        main([case_path("pd_coarse.json"), "--surrogate", "fast"])
    assert not (tmp_path / "o").exists()


def test_initial_state_loads():
    """initialState and its overrides give every point's starting state (DemoConfig.cpp:220-251)."""
    with open(case_path("pd_coarse.json")) as f:
        d = json.load(f)
    d["materials"][0].update(initialStateOverrides={"1": 0.01, "2": 300.0})
    import tempfile
    with tempfile.TemporaryDirectory() as t:
        p = os.path.join(t, "case.json")
        with open(p, "w") as f:
            json.dump(d, f)
        m = load_boundary_case(p, golden("")).materials[0]
    assert m.initial_state == (0.0, 0.01, 300.0, 0.0, 0.0, 0.0)
    assert load_boundary_case(case_path("pd_coarse.json"), golden("")).materials[0].initial_state == ()


def test_internal_indicator_values():
    """internalIndicator (BoundaryValueCaseRunner.cpp:93-107): min or max over the chosen state
    variables, NaN skipped as std::min/std::max skip their second argument, then one_minus;
    no clamp at 0 here (the per-step maximum starts at 0 on the device)."""
    from vpd.boundary_case import indicator_values
    state = np.array([[0.0, 0.2, 0.5], [0.0, np.nan, 0.1], [0.0, -0.3, -0.1]])
    assert np.allclose(indicator_values(((1, 2), "max", "identity"), state), [0.5, 0.1, -0.1])
    assert np.allclose(indicator_values(((1, 2), "min", "one_minus"), state), [0.8, 0.9, 1.3])
    assert np.array_equal(indicator_values(None, state), np.zeros(3))
    with open(case_path("pd_coarse.json")) as f:
        d = json.load(f)
    d["materials"][0]["internalIndicator"] = {"indices": [1], "reduction": "max"}
    import tempfile
    with tempfile.TemporaryDirectory() as t:
        p = os.path.join(t, "case.json")
        with open(p, "w") as f:
            json.dump(d, f)
        assert load_boundary_case(p, golden("")).materials[0].indicator == ((1,), "max", "identity")
