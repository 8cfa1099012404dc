"""The point damage modes (SimpleDamageModel::update / degradeStress, SimpleDamageModel.cpp:14-50,
as PdSimpleDamage.cpp:84-92 runs them) on the device, against the oracle, which reproduces the
reference library's own damage modules bit for bit on these cases (test_oracle.py).

pd_coarse through 2400 increments: the thresholds are crossed in the necking band, so part of
the bar is fully damaged and part untouched. Tolerances as the other full-run parity tests:
NRMSE <= 1e-6 on the stress timeseries and the fields."""
import os

import numpy as np
import pytest

from conftest import nrmse

import oracle as O
import vpd
from vpd.case import (DAMAGE_EQPS_THRESHOLD, DAMAGE_MAX_PRINCIPAL_STRAIN, MATERIAL_SURROGATE,
                      PRECISION_MIXED, pd_coarse)

pytestmark = pytest.mark.gpu

STRESS = vpd.DIAG["average_axial_stress_MPa"]
POINT_DAMAGE = [(DAMAGE_EQPS_THRESHOLD, 0.002, 0.03, False), (DAMAGE_EQPS_THRESHOLD, 0.001, 0.01, True),
                (DAMAGE_MAX_PRINCIPAL_STRAIN, 0.005, 0.03, False)]
FIELDS = ("displacement", "velocity", "stress_corotational", "state", "damage_index")


def damaged(mode, initiation, failure, deletion, **kw):
    return pd_coarse().replace(steps=2400, damage_mode=mode, damage_initiation=initiation,
                               damage_failure=failure, damage_deletion=deletion, **kw)


def run(case, plugin=None):
    with vpd.Simulation(case) as sim:
        if plugin:
            sim.set_host_vumat(plugin, case.props, case.nstatev, case.props[10])
        rows = sim.step(case.steps)
        return rows, {f: sim.field(f) for f in FIELDS}


@pytest.mark.parametrize("mode, initiation, failure, deletion", POINT_DAMAGE)
def test_point_damage_matches_oracle(mode, initiation, failure, deletion):
    case = damaged(mode, initiation, failure, deletion)
    rows, f = run(case)
    o = O.OracleSim(case)
    ref = o.step(case.steps)
    assert nrmse(rows[:, STRESS], ref[:, STRESS]) < 1e-6
    for name in FIELDS:
        a, b = f[name], o.get(name)
        if name == "state":  # not variable 6, the JC's running count of bisection iterations
            a, b = a[:, :5], b[:, :5]
        assert nrmse(a, b) < 1e-6, name
    d = f["damage_index"]
    assert (d >= 1.0).sum() > 100 and (d == 0.0).sum() > 100


def test_point_damage_through_host_plugin():
    """The host VUMAT path applies the same damage: the JC plugin against the device update."""
    case = damaged(*POINT_DAMAGE[1])
    ra, fa = run(case)
    rb, fb = run(case, os.path.join(O.REF_DIR, "jc_vumat_plugin.so"))
    assert nrmse(rb[:, STRESS], ra[:, STRESS]) < 1e-9
    for name in FIELDS:
        a, b = fb[name], fa[name]
        if name == "state":  # not variable 6, the JC's running count of bisection iterations
            a, b = a[:, :5], b[:, :5]
        assert nrmse(a, b) < 1e-8, name


def test_point_damage_mixed_precision():
    """FP32 bond sums with the point damage: close to the FP64 run."""
    case = damaged(*POINT_DAMAGE[0])
    ra, fa = run(case)
    rb, fb = run(case.replace(precision=PRECISION_MIXED))
    assert np.isfinite(rb).all()
    assert nrmse(rb[:, STRESS], ra[:, STRESS]) < 1e-3
    assert nrmse(fb["damage_index"], fa["damage_index"]) < 1e-2


def test_point_damage_errors():
    with pytest.raises(vpd.VpdError, match="requires failure > initiation"):
        vpd.Simulation(damaged(DAMAGE_EQPS_THRESHOLD, 0.01, 0.01, False))
    with pytest.raises(vpd.VpdError, match="VPD_MATERIAL_VUMAT"):
        vpd.Simulation(damaged(*POINT_DAMAGE[0], material_mode=MATERIAL_SURROGATE))
    case = damaged(*POINT_DAMAGE[0])
    with vpd.Simulation(case) as sim:
        with pytest.raises(vpd.VpdError, match="eqpsStateIndex is outside the VUMAT state vector"):
            sim.set_host_vumat(os.path.join(O.REF_DIR, "jc_vumat_plugin.so"), case.props, 1, 7800.0)
