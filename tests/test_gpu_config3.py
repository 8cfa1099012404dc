"""The physics of the 1M-point benchmark bar (400x50x50, +-0.05 h jitter, horizon 4.015 h,
about 238 bonds per point, Johnson-Cook with adiabatic heating (workToHeat 1e6), grips at
5 m/s, critical stretch 0.02) on the GPU against the reference library.

* A 24-plane slab of that bar (24x50x50 = 60,000 points: the full cross-section, the same
  horizon, jitter stream, heating, grips and damage) against the reference library's own run
  of it (fixture ref_config3_slab.npz, made by tests/golden/make_golden.py --config3 with
  oracle/_ref, the reference's C++ compiled from its sources): 160 increments, through the
  first broken bonds (from increment ~90) and into yield (~140). The plain FP64 path on its
  default tiled kernels: stress history NRMSE <= 1e-6, displacements within 1e-9, the damage
  index of every point identical, JC iteration counts equal on > 99.9 % of points. The mixed
  and surrogate + mixed paths: stress NRMSE <= 0.5 %, damage indices equal on > 99.9 % of
  points.
* The whole bar with its specified damage fails progressively: bonds first break near the
  grips, and the broken fraction then grows until the bar has come apart, while the same bar
  without damage stays intact and flows plastically. The reference library shows the same
  cascade on the slab (tests/test_oracle.py::test_reference_library_config3_slab_cascades).
"""
import numpy as np
import pytest

from conftest import golden, max_rel, nrmse

import vpd
from vpd.case import MATERIAL_SURROGATE, PRECISION_FP64, PRECISION_MIXED, tensile_bar

pytestmark = pytest.mark.gpu

STRESS = vpd.DIAG["average_axial_stress_MPa"]
SLAB_STEPS = 160


@pytest.fixture(scope="module")
def ref():
    return np.load(golden("ref_config3_slab.npz"))


def slab(precision=PRECISION_FP64, **kw):
    return tensile_bar(3, nx=24, precision=precision, **kw)


def run_slab(case, surrogate=None):
    with vpd.Simulation(case) as sim:
        if surrogate is not None:
            sim.set_surrogate(*surrogate, guess="hybrid", newton_steps=2)
        rows = sim.step(SLAB_STEPS)
        fields = {f: sim.field(f) for f in ("displacement", "stress_corotational", "state",
                                            "damage_index")}
    return rows, fields


def test_config3_slab_fp64_matches_reference_library(ref):
    rows, f = run_slab(slab())
    pick = np.arange(0, len(f["damage_index"]), int(ref["stride"]))
    d_ref = ref["damage_index"]
    assert (d_ref > 0).sum() > 10000 and ref["diag"][-1, vpd.DIAG["plastic_points"]] > 10000
    assert nrmse(rows[:, STRESS], ref["diag"][:, STRESS]) < 1e-6
    for c in ("reaction_force_N", "max_eqps", "kinetic_energy_Nmm", "internal_energy_Nmm",
              "external_work_Nmm", "average_axial_strain"):
        assert max_rel(rows[:, vpd.DIAG[c]], ref["diag"][:, vpd.DIAG[c]]) < 1e-8, c
    assert np.array_equal(f["damage_index"][:, 0], d_ref)
    assert max_rel(f["displacement"][pick], ref["displacement"]) < 1e-9
    sigma = f["stress_corotational"][pick][:, [0, 4, 8, 1, 5, 2]]
    assert max_rel(sigma, ref["stress_corotational6"]) < 1e-8
    assert max_rel(f["state"][pick][:, 1], ref["state"][:, 0]) < 1e-8  # eqps
    assert np.mean(f["state"][pick][:, 5] == ref["state"][:, 1]) > 0.999  # JC iterations


@pytest.mark.parametrize("mode", ["mixed", "surrogate_mixed"])
def test_config3_slab_mixed_paths_against_reference_library(ref, mode):
    surrogate = None
    case = slab(PRECISION_MIXED)
    if mode == "surrogate_mixed":
        case = case.replace(material_mode=MATERIAL_SURROGATE)
        w, b, _ = vpd.train_surrogate(case.props, samples=262144, epochs=4)
        surrogate = (w, b)
    rows, f = run_slab(case, surrogate)
    assert nrmse(rows[:, STRESS], ref["diag"][:, STRESS]) < 5e-3
    assert np.mean(f["damage_index"][:, 0] == ref["damage_index"]) > 0.999
    pick = np.arange(0, len(f["damage_index"]), int(ref["stride"]))
    u_ref = ref["displacement"]
    assert np.sqrt(np.mean((f["displacement"][pick] - u_ref) ** 2)) / np.abs(u_ref).max() < 5e-3


def test_config3_bar_with_damage_comes_apart():
    """The whole 1M-point bar as specified (critical stretch 0.02), plain FP64: its first bonds
    break between increments 100 and 200, near the grips and before the bar yields; by
    increment 800 nine tenths of all bonds are broken and the equivalent plastic strain has run
    away (the correspondence F keeps summing over broken bonds). Without damage the same bar
    stays intact and flows plastically (the benchmark's headline workload)."""
    S = vpd.DIAG
    case = tensile_bar(3, precision=PRECISION_FP64)
    first = None
    with vpd.Simulation(case) as sim:
        for done in range(25, 801, 25):
            rows = sim.step(25)
            d = sim.field("damage_index")[:, 0]
            if first is None and d.max() > 0:
                first = done
                assert rows[-1, S["plastic_points"]] == 0  # breaks before anything yields
        assert 100 < first <= 200
        assert d.mean() > 0.9 and np.mean(d > 0) > 0.999
        assert rows[-1, S["max_eqps"]] > 1.0
    with vpd.Simulation(case.replace(damage_mode=0)) as sim:
        rows = sim.step(800)
        assert np.all(rows[:, S["finite"]] == 1.0)
        assert 0 < rows[-1, S["max_eqps"]] < 0.05
        assert rows[-1, S["plastic_points"]] > 1000
