"""Checkpoint and resume (vpd_checkpoint_save / vpd_checkpoint_load): a simulation restored
from a checkpoint continues bit for bit as the saved one does, on every bond layout,
precision and material path; a checkpoint of another case is refused."""
import os

import numpy as np
import pytest

import oracle as O
import vpd
from vpd.case import (DAMAGE_CRITICAL_STRETCH, DAMAGE_EQPS_THRESHOLD, MATERIAL_SURROGATE,
                      PRECISION_MIXED, pd_coarse, tensile_bar)

pytestmark = pytest.mark.gpu

FIELDS = ("displacement", "velocity", "acceleration", "stress_corotational", "state",
          "damage_index", "temperature")


def jc_plugin(sim, case):
    sim.set_host_vumat(os.path.join(O.REF_DIR, "jc_vumat_plugin.so"), case.props, case.nstatev,
                       case.props[10])


CASES = {
    "fp64_stencil_damage": (tensile_bar(1, jitter=0.05, jitter_seed=7, damage_mode=DAMAGE_CRITICAL_STRETCH,
                                        damage_initiation=0.004), None, {}),
    "fp64_ell_damage": (tensile_bar(1, jitter=0.05, jitter_seed=7, damage_mode=DAMAGE_CRITICAL_STRETCH,
                                    damage_initiation=0.004), None, {"VPD_BOND_LAYOUT": "ell"}),
    "mixed": (tensile_bar(1, precision=PRECISION_MIXED, damage_mode=DAMAGE_CRITICAL_STRETCH,
                          damage_initiation=0.004), None, {}),
    "point_damage": (pd_coarse().replace(damage_mode=DAMAGE_EQPS_THRESHOLD, damage_initiation=1e-4,
                                         damage_failure=2e-3, damage_deletion=True), None, {}),
    "host_plugin": (pd_coarse(), jc_plugin, {}),
    "surrogate_warm": (tensile_bar(1, material_mode=MATERIAL_SURROGATE), "warm", {}),
}


def setup(sim, case, how):
    if how == "warm":
        sim.set_surrogate(guess="warm_start", newton_steps=2)
    elif how is not None:
        how(sim, case)


@pytest.mark.parametrize("name", sorted(CASES))
def test_resume_continues_bit_for_bit(monkeypatch, name):
    case, how, env = CASES[name]
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    with vpd.Simulation(case) as a:
        setup(a, case, how)
        a.step(700)
        saved = a.checkpoint()
        rows_a = a.step(300)
        fa = {f: a.field(f) for f in FIELDS}
    with vpd.Simulation(case) as b:
        setup(b, case, how)
        b.restore(saved)
        rows_b = b.step(300)
        for f in FIELDS:
            assert np.array_equal(b.field(f), fa[f]), f
    assert np.array_equal(rows_a, rows_b)
    assert rows_b[0, vpd.DIAG["step"]] == 701


def test_checkpoint_of_another_case_is_refused():
    with vpd.Simulation(pd_coarse()) as a:
        a.step(3)
        saved = a.checkpoint()
    with vpd.Simulation(pd_coarse().replace(dt=pd_coarse().dt * 0.5)) as b:
        with pytest.raises(vpd.VpdError, match="another case"):
            b.restore(saved)
        with pytest.raises(vpd.VpdError, match="not a checkpoint"):
            b.restore(b"x" * len(saved))
    with vpd.Simulation(pd_coarse()) as c:
        with pytest.raises(vpd.VpdError, match="size"):
            c.restore(saved[:-8])
        c.restore(saved)
        assert c.step(1)[0, vpd.DIAG["step"]] == 4
