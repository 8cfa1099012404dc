"""The certified Johnson-Cook return map (jc_return_map) against the VUMAT's literal bisection
(jc_bisection, JohnsonCook.f90:114-136): the same plastic increment, yield stress and iteration
count, bit for bit.

* vpd_jc_return_map on two million random states through the C ABI: elastic and plastic
  trials, first yield (no previous increment to start from), warm starts on either side of
  the root, an old yield stress of zero, temperatures up to the melting point (a vanishing
  thermal factor), increments large enough to clip the new equivalent stress at zero, tiny
  increments whose rate term is negative, points on their initialising call and non-finite
  inputs.
* Whole increments on a slab of the benchmark bar (the 24x50x50 slab of tensile_bar(3):
  horizon 4.015 h, jitter, adiabatic heating, grips at 5 m/s) run into yield with the
  material kernel on each return map (VPD_RETURN_MAP=bisection selects the literal one): the
  diagnostics rows and every field are identical, in FP64 and in mixed precision.
"""
import numpy as np
import pytest

import vpd
from vpd.case import PRECISION_FP64, PRECISION_MIXED, tensile_bar

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def random_states(n, seed):
    """Old stress, state and strain increments spanning the regimes the return map meets."""
    rng = np.random.default_rng(seed)
    stress = rng.standard_normal((n, 6)) * rng.choice([30.0, 300.0, 900.0], size=(n, 1))
    eqps = 10.0 ** rng.uniform(-6, np.log10(0.5), n)
    eqps[rng.random(n) < 0.05] = 0.0
    temp = rng.uniform(293.0, 1793.0, n)
    temp[rng.random(n) < 0.02] = 1793.0  # at the melting point: thermal factor 0
    old_yield = rng.uniform(200.0, 900.0, n)
    old_yield[rng.random(n) < 0.1] = 0.0
    warm = 10.0 ** rng.uniform(-10, -2, n)
    warm[rng.random(n) < 0.2] = 0.0
    state = np.column_stack([np.ones(n), eqps, temp, old_yield, warm, np.zeros(n)])
    state[rng.random(n) < 0.01, 0] = 0.0  # initialising call
    scale = 10.0 ** rng.uniform(-7, -1.5, (n, 1))
    inc = rng.standard_normal((n, 6)) * scale
    # a share of the increments along the old stress deviator (steady plastic flow)
    along = rng.random(n) < 0.4
    dev = stress.copy()
    dev[:, :3] -= dev[:, :3].mean(axis=1, keepdims=True)
    inc[along] = dev[along] / (np.linalg.norm(dev[along], axis=1, keepdims=True) + 1e-30) * scale[along]
    bad = rng.random(n) < 1e-4
    stress[bad, 0] = np.nan
    inc[rng.random(n) < 1e-4, 2] = np.inf
    return inc, stress, state


@pytest.mark.parametrize("dt", [tensile_bar(3, nx=8).dt, tensile_bar(1).dt])
def test_certified_return_map_matches_literal_bisection(dt):
    props = tensile_bar(3, nx=8).props
    inc, stress, state = random_states(1 << 21, seed=11)
    args = [torch.from_numpy(a).cuda() for a in (inc, stress, state)]
    fast = [t.cpu().numpy() for t in vpd.jc_return_map(props, dt, *args, method=0)]
    literal = [t.cpu().numpy() for t in vpd.jc_return_map(props, dt, *args, method=1)]
    plastic = literal[2] > 1
    assert plastic.mean() > 0.3 and (literal[2] == 1).mean() > 0.05
    assert (literal[2] >= 20).sum() > 1000  # long bisections, where the certified one saves most
    for name, f, l in zip(("ep_inc", "yield", "iterations"), fast, literal):
        assert same_bits(f, l), (name, np.flatnonzero(~((f == l) | (np.isnan(f) & np.isnan(l))))[:10])


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED])
def test_increments_identical_with_literal_bisection(monkeypatch, precision):
    case = tensile_bar(3, nx=24, precision=precision)
    fields = ("displacement", "velocity", "stress_corotational", "state", "damage_index")

    def run():
        with vpd.Simulation(case) as sim:
            rows = sim.step(220)
            return rows, {f: sim.field(f) for f in fields}

    rows_c, f_c = run()
    monkeypatch.setenv("VPD_RETURN_MAP", "bisection")
    rows_l, f_l = run()
    assert rows_l[-1, vpd.DIAG["plastic_points"]] > 10000
    assert same_bits(rows_c, rows_l)
    for f in fields:
        assert same_bits(f_c[f], f_l[f]), f
