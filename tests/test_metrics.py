"""The restated PD analysis metrics (vpd.metrics, analyse_and_plot.py:44-82) pinned to the
reference's frozen values (expected/analysis.json): computed from the archived PD runs and
the archived FEM reference (fixtures written by tests/golden/make_golden.py --archived), every
PD case's metrics must equal the frozen ones far inside verify_metrics.py's 0.5 %."""
import json
import math

import numpy as np
import pytest

from conftest import golden

from vpd import metrics as VM

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


def archived_series(data, name):
    cols = [str(c) for c in data[f"{name}_columns"]]
    return {c: data[f"{name}_timeseries"][:, j] for j, c in enumerate(cols)}


def test_sample_coordinates():
    c = VM.sample_coordinates()
    assert c.shape == (1551, 3)
    assert np.array_equal(c[0], [4.0, -10.0, -2.0]) and np.array_equal(c[-1], [96.0, 10.0, 2.0])
    assert np.array_equal(c[1], [4.0, -10.0, 0.0])


def test_trilinear_interpolation_is_exact_for_affine_fields():
    x, y, z = np.meshgrid(np.arange(0.0, 101.0, 2.0), np.arange(-10.0, 11.0, 2.0),
                          np.arange(-2.0, 3.0, 2.0), indexing="ij")
    nodes = {"x0_mm": x.ravel(), "y0_mm": y.ravel(), "z0_mm": z.ravel()}
    nodes["ux_mm"] = 0.01 * nodes["x0_mm"] + 0.2
    nodes["uy_mm"] = -0.003 * nodes["y0_mm"] + 0.001 * nodes["x0_mm"]
    nodes["uz_mm"] = 0.002 * nodes["z0_mm"]
    rng = np.random.default_rng(1)
    perm = rng.permutation(len(nodes["x0_mm"]))  # row order must not matter
    nodes = {k: v[perm] for k, v in nodes.items()}
    q = VM.sample_coordinates() + rng.uniform(-0.9, 0.9, (1551, 3)) * [1, 1, 0]
    q[:, 1] = np.clip(q[:, 1], -10.0, 10.0)
    u = VM.interpolate_nodes(nodes, q)
    exact = np.stack([0.01 * q[:, 0] + 0.2, -0.003 * q[:, 1] + 0.001 * q[:, 0], 0.002 * q[:, 2]], 1)
    assert np.max(np.abs(u - exact)) < 1e-14


@pytest.mark.parametrize("name", CASES)
def test_metrics_of_archived_runs_equal_frozen_values(archive, name):
    data, expected, ref = archive
    series = archived_series(data, name)
    got = VM.pd_metrics(series, data[f"{name}_u"], expected[name]["nodes"], ref)
    assert set(got) == set(expected[name])
    for k, v in expected[name].items():
        assert math.isclose(got[k], v, rel_tol=1e-9, abs_tol=1e-12), (k, got[k], v)
    assert VM.mismatches(expected[name], got) == []
    # a run 1 % off in stress fails the reference's 0.5 % check
    off = dict(series, average_axial_stress_MPa=series["average_axial_stress_MPa"] * 1.01)
    assert "stress_MPa" in VM.mismatches(expected[name], VM.pd_metrics(off, data[f"{name}_u"], 0, ref))
