"""The material update through a host VUMAT plugin (vpd_set_host_vumat): the reference's
VUMAT-PD bridge (src/material/VumatPdCorrespondenceMaterial.cpp:72-176 with
src/material/VumatMaterialAdapter.cpp:147-362) fed by the device increment.

Checked against two references: the device Johnson-Cook update, with the plugin being the C
restatement of the Fortran JC routine; and the reference library's own modules (RefSim) running
the linear-elastic plugin. Every case has a short last block (1683 = 6 x 256 + 147 and
4000 = 15 x 256 + 160 points), so the padding of the last plugin call is exercised.
Tolerances as the device-update parity tests: stress NRMSE <= 1e-9 on the timeseries, fields
within 1e-8 relative."""
import os

import numpy as np
import pytest

from conftest import max_rel, nrmse

import oracle as O
import vpd
from vpd.case import MATERIAL_SURROGATE, PRECISION_MIXED, pd_coarse, tensile_bar

pytestmark = pytest.mark.gpu

STRESS = vpd.DIAG["average_axial_stress_MPa"]
JC_PLUGIN = os.path.join(O.REF_DIR, "jc_vumat_plugin.so")
ELASTIC_PLUGIN = os.path.join(O.REF_DIR, "elastic_vumat_plugin.so")


def attach(sim, case, plugin, **kw):
    sim.set_host_vumat(plugin, case.props, case.nstatev, case.props[10], **kw)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_host_jc_plugin_matches_device_update(precision):
    """The 40x10x10 bar into plastic flow: the JC plugin on the host gives the device update's
    increments (the plugin and the device routine agree to 1e-12 on single blocks)."""
    extra = dict(precision=PRECISION_MIXED) if precision == "mixed" else {}
    case = tensile_bar(1, **extra)
    steps = 2000 if precision == "fp64" else 600
    fields = ("displacement", "velocity", "stress_corotational", "state")
    with vpd.Simulation(case) as a:
        ra = a.step(steps)
        fa = {f: a.field(f) for f in fields}
    with vpd.Simulation(case) as b:
        attach(b, case, JC_PLUGIN)
        rb = b.step(steps)
        fb = {f: b.field(f) for f in fields}
        temperature = b.field("temperature")
    if precision == "fp64":
        assert ra[-1, vpd.DIAG["max_eqps"]] > 1e-3
    # mixed: FP32 bond sums carry the plugin's last-bit differences further (stress ~2e-9,
    # velocities ~1e-6)
    tol = 1e-8 if precision == "fp64" else 1e-5
    assert nrmse(rb[:, STRESS], ra[:, STRESS]) < (1e-9 if precision == "fp64" else 1e-7)
    for f in ("displacement", "velocity", "stress_corotational"):
        assert nrmse(fb[f], fa[f]) < tol, f
    assert nrmse(fb["state"][:, 1], fa["state"][:, 1]) < tol
    assert np.isfinite(temperature).all() and temperature.min() >= case.reference_temperature


@pytest.mark.skipif(not O.reference_available(), reason="reference library not built")
def test_host_elastic_plugin_matches_reference_library():
    """pd_coarse with the linear-elastic plugin: the device increment around the host plugin
    against the reference's own bridge, adapter and modules running the same plugin."""
    case = pd_coarse().replace(steps=600)
    ref = O.RefSim(case, plugin="elastic_vumat_plugin.so")
    rr = ref.step(600)
    with vpd.Simulation(case) as sim:
        attach(sim, case, ELASTIC_PLUGIN)
        rows = sim.step(600)
        assert nrmse(rows[:, STRESS], rr[:, STRESS]) < 1e-9
        assert max_rel(sim.field("displacement"), ref.get("displacement")) < 1e-8
        assert nrmse(sim.field("stress_corotational"), ref.get("stress_corotational")) < 1e-8
        assert np.all(sim.field("state") == 0.0)  # the elastic routine copies its state
        assert np.all(sim.field("temperature") == case.reference_temperature)
    assert rows[-1, vpd.DIAG["max_eqps"]] == 0.0


def test_host_plugin_graph_and_stage_launches_agree_bitwise():
    """The plugin's copies and host function are captured in the increment's CUDA graph: graph
    replays and launch-by-launch increments give the same bits."""
    case = pd_coarse().replace(steps=64)
    with vpd.Simulation(case) as a, vpd.Simulation(case) as b:
        attach(a, case, JC_PLUGIN)
        attach(b, case, JC_PLUGIN)
        a.step(40)
        b.profile_stages(40)
        for f in ("displacement", "velocity", "stress_corotational", "state", "temperature"):
            assert np.array_equal(a.field(f), b.field(f)), f


def test_host_plugin_errors():
    """The adapter's construction errors, with its messages, and the handle-level checks."""
    case = pd_coarse()
    with vpd.Simulation(case) as sim:
        with pytest.raises(vpd.VpdError, match="Failed to load VUMAT plugin"):
            attach(sim, case, os.path.join(O.REF_DIR, "no_such_plugin.so"))
        with pytest.raises(vpd.VpdError, match="Failed to resolve symbol in VUMAT plugin: vumat_nope"):
            attach(sim, case, JC_PLUGIN, symbol="vumat_nope")
        with pytest.raises(vpd.VpdError, match="VUMAT props cannot be empty"):
            sim.set_host_vumat(JC_PLUGIN, [], 6, 7800.0)
        with pytest.raises(vpd.VpdError, match="nstatev must be non-negative"):
            sim.set_host_vumat(JC_PLUGIN, case.props, -1, 7800.0)
        with pytest.raises(vpd.VpdError, match="exceeds the case's nstatev"):
            sim.set_host_vumat(JC_PLUGIN, case.props, case.nstatev + 1, 7800.0)
        attach(sim, case, JC_PLUGIN)
        with pytest.raises(vpd.VpdError, match="already attached"):
            attach(sim, case, JC_PLUGIN)
    with vpd.Simulation(case) as sim:
        sim.step(1)
        with pytest.raises(vpd.VpdError, match="before the first vpd_step"):
            attach(sim, case, JC_PLUGIN)
    sc = case.replace(material_mode=MATERIAL_SURROGATE)
    with vpd.Simulation(sc) as sim:
        with pytest.raises(vpd.VpdError, match="not VPD_MATERIAL_VUMAT"):
            attach(sim, sc, JC_PLUGIN)
