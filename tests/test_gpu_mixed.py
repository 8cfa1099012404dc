"""Mixed precision (FP32 bond sums with Kahan-folded partials, FP64 kinematics, return map and
integration) against the plain FP64 path on the same case. The stated tolerance is stress
history NRMSE <= 0.5 %; displacement and equivalent plastic strain errors are checked too."""
import numpy as np
import pytest

from conftest import nrmse

import vpd
from vpd.case import PRECISION_FP64, PRECISION_MIXED, tensile_bar

pytestmark = pytest.mark.gpu

STRESS = vpd.DIAG["average_axial_stress_MPa"]
TOL = 5e-3  # stress-history NRMSE bound for the mixed and surrogate forms


def run(case, steps):
    with vpd.Simulation(case) as sim:
        rows = sim.step(steps)
        return rows, sim.field("displacement"), sim.field("state")[:, 1], sim.field("damage_index")


def test_mixed_tracks_fp64_full_tensile_bar_1():
    """The 40x10x10 bar over its 2000 increments, into the plastic range."""
    case = tensile_bar(1)
    r64, u64, ep64, _ = run(case.replace(precision=PRECISION_FP64), case.steps)
    r32, u32, ep32, _ = run(case.replace(precision=PRECISION_MIXED), case.steps)
    assert ep64.max() > 1e-3
    s_err = nrmse(r32[:, STRESS], r64[:, STRESS])
    assert s_err < TOL
    assert s_err < 1e-4  # observed ~1e-6
    assert nrmse(u32, u64) < 1e-4
    assert nrmse(ep32, ep64) < 1e-2


def test_mixed_tracks_fp64_jittered_horizon_4():
    """The 1M-point bar's cross-section and horizon (jitter +-0.05 h, delta 4.015 h), 60
    planes long, 1500 increments without damage (plastic at the grips)."""
    case = tensile_bar(3, nx=60, damage_mode=0)
    r64, u64, ep64, _ = run(case.replace(precision=PRECISION_FP64), 1500)
    r32, u32, ep32, _ = run(case.replace(precision=PRECISION_MIXED), 1500)
    assert ep64.max() > 1e-3
    assert nrmse(r32[:, STRESS], r64[:, STRESS]) < TOL
    assert nrmse(u32, u64) < 1e-3
    assert nrmse(ep32, ep64) < 5e-2


def test_mixed_damage_decisions_match_fp64_early():
    """Bond breaking in FP32 falls back to the exact FP64 test near the threshold: over the
    first increments of a damaged jittered bar the broken-bond fractions agree."""
    case = tensile_bar(1, jitter=0.05, jitter_seed=7, damage_mode=1, damage_initiation=0.004)
    r64, _, _, d64 = run(case.replace(precision=PRECISION_FP64), 120)
    r32, _, _, d32 = run(case.replace(precision=PRECISION_MIXED), 120)
    assert d64.max() > 0
    assert np.mean(np.abs(d32 - d64) < 1e-12) > 0.99
    assert nrmse(r32[:, STRESS], r64[:, STRESS]) < TOL


def test_thin_lattice_windows_reach_past_both_ends(monkeypatch):
    """A lattice thinner than the stencil (8 x 3 x 5 points, horizon 4.015 h, jittered): the
    packed kernels' windows reach several planes past every end of the lattice, into the zero
    halos of their neighbour arrays, while the per-slot kernels clamp every index. Both must
    give the same increments to FP32 rounding, and the mixed run must track FP64."""
    case = tensile_bar(3, nx=8, ny=3, nz=5, damage_mode=0, precision=PRECISION_MIXED)
    monkeypatch.setenv("VPD_BOND_KERNEL", "slot")
    rs, us, _, _ = run(case, 300)
    monkeypatch.setenv("VPD_BOND_KERNEL", "pair")
    rp, up, _, _ = run(case, 300)
    assert np.all(np.isfinite(rp)) and np.all(np.isfinite(up))
    assert nrmse(rp[:, STRESS], rs[:, STRESS]) < 1e-5
    assert nrmse(up, us) < 1e-5
    monkeypatch.delenv("VPD_BOND_KERNEL")
    r64, u64, _, _ = run(case.replace(precision=PRECISION_FP64), 300)
    assert nrmse(rp[:, STRESS], r64[:, STRESS]) < 1e-4
    assert nrmse(up, u64) < 1e-4


def test_mixed_requires_lattice_layout(monkeypatch):
    monkeypatch.setenv("VPD_BOND_LAYOUT", "ell")
    with pytest.raises(vpd.VpdError) as e:
        vpd.Simulation(tensile_bar(1, precision=PRECISION_MIXED))
    assert e.value.status == 6


@pytest.mark.parametrize("damage", [0, 1])
def test_tiled_bond_kernels_match_slot_kernels(monkeypatch, damage):
    """The tiled bond kernels (two points per thread along y, one load per neighbour record
    per stencil group; scalar FP32 and packed FP32 pairs) against the per-slot kernels on the
    jittered horizon-4 bar: the same FP32 bond terms summed in another order, so the histories
    agree to FP32 rounding and the bond-breaking decisions agree. With damage the comparison covers the early increments:
    later, rounding-level differences flip bonds at the threshold and the fracture paths part
    (as between the FP64 and mixed paths)."""
    case = tensile_bar(3, nx=24, ny=20, nz=17, damage_mode=damage, damage_initiation=0.004,
                       precision=PRECISION_MIXED)
    steps = 120 if damage else 400
    monkeypatch.setenv("VPD_BOND_KERNEL", "slot")
    rs, us, es, ds = run(case, steps)
    for kind in ("scalar", "pair"):
        monkeypatch.setenv("VPD_BOND_KERNEL", kind)
        rt, ut, et, dt_ = run(case, steps)
        assert nrmse(rt[:, STRESS], rs[:, STRESS]) < 1e-5
        assert nrmse(ut, us) < 1e-5
        if damage:
            assert ds.max() > 0
            assert np.mean(np.abs(dt_ - ds) < 1e-12) > 0.99
