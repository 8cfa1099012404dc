"""The material-point case host (vpd.point_runner) on CPU, against the reference's own CLI.

The reference's vumat_pd_run (oracle/_ref, built from its sources) and this runner both load the
same plugin library (the restated Johnson-Cook or elastic routine in oracle/_ref) and run the
same case file, so their output files must agree byte for byte: that pins the host logic (the
loading path, the plane-strain bisection, the adapter's argument packing, the writers). The
stock path, with the Johnson-Cook routine on the GPU, is checked in test_gpu_point_runner.py."""
import gzip
import json
import os
import shutil
import subprocess

import pytest

from conftest import golden

import oracle as O
from vpd.point_runner import load_point_case, run_material_point_case

CLI = os.path.join(O.REF_DIR, "vumat_pd_run")
needs_cli = pytest.mark.skipif(not os.path.exists(CLI), reason="reference CLI not built")


def fixture(case, name):
    with gzip.open(golden(os.path.join("example_outputs", case, name + ".gz")), "rb") as f:
        return f.read()


def test_jc_material_point_reproduces_reference_output(tmp_path):
    """examples/jc_material_point.json (plane strain, uniaxial stress by bisection, 600 steps)
    against the reference CLI's files stored in tests/golden/example_outputs."""
    rc = run_material_point_case(golden("examples/jc_material_point.json"), str(tmp_path),
                                 config_root=golden(""), plugin_dir=O.REF_DIR, log=lambda *a: None)
    assert rc == 0
    for name in ("timeseries.csv", "metadata.json"):
        assert (tmp_path / name).read_bytes() == fixture("jc_material_point", name), name


def test_bisection_tree_blocks_reproduce_reference_output(tmp_path):
    """The plane-strain bisection evaluated 8 levels per plugin call (the GPU library's
    setting) with the restated plugin: the same bytes as the reference CLI's sequential run."""
    rc = run_material_point_case(golden("examples/jc_material_point.json"), str(tmp_path),
                                 config_root=golden(""), plugin_dir=O.REF_DIR, log=lambda *a: None,
                                 tree_levels=8)
    assert rc == 0
    for name in ("timeseries.csv", "metadata.json"):
        assert (tmp_path / name).read_bytes() == fixture("jc_material_point", name), name


def reference_cli(tmp_path, case):
    """Runs the reference CLI on a case dict; returns its output directory."""
    work = tmp_path / "ref"
    shutil.copytree(golden("configs"), work / "configs")
    (work / "examples").mkdir()
    case = dict(case, output={"directory": "out"})
    (work / "examples" / "case.json").write_text(json.dumps(case))
    subprocess.run([CLI, "examples/case.json"], cwd=work, check=True, stdout=subprocess.DEVNULL)
    return work / "out", work / "examples" / "case.json"


@needs_cli
@pytest.mark.parametrize("mode, config, reference", [
    ("uniaxial_xx", "configs/elastic.json", True),
    ("simple_shear_xy", "configs/elastic.json", True),
    ("simple_shear_xy", "configs/johnson_cook.json", False),
    ("uniaxial_xx", "configs/johnson_cook.json", False),
])
def test_point_modes_match_reference_cli(tmp_path, mode, config, reference):
    with open(golden("examples/jc_material_point.json")) as f:
        case = json.load(f)
    case["boundary_conditions"] = {"type": "affine_displacement", "mode": mode, "maxStrain": 0.03}
    case["time_integration"].update(steps=120, totalTime=120 * case["time_integration"]["dt"])
    case["materials"][0].update(materialConfigPath=config, reference=reference)
    if "elastic" in config:  # one state variable
        case["materials"][0].update(equivalentPlasticStrainIndex=0, internalIndicator={"indices": [0]})
    case["tolerances"] = {"referenceStressAbsolute": 1e-6}
    ref_out, path = reference_cli(tmp_path, case)
    ours = tmp_path / "ours"
    rc = run_material_point_case(str(path), str(ours), config_root=str(path.parent.parent),
                                 plugin_dir=O.REF_DIR, log=lambda *a: None)
    for name in ("timeseries.csv", "metadata.json"):
        assert (ours / name).read_bytes() == (ref_out / name).read_bytes(), name
    assert rc == (0 if json.loads((ours / "metadata.json").read_text())["status"] == "pass" else 2)


def test_point_case_loading():
    case = load_point_case(golden("examples/jc_material_point.json"), golden(""))
    assert (case.steps, case.dt, case.mode) == (600, 0.0002, "plane_strain_x_uniaxial_stress")
    m = case.materials[0]
    assert m.config.cmname == "JOHNSONCOOK" and m.config.nstatev == 6 and m.config.nfieldv == 1
    assert m.indicator_indices == [1] and m.reference_temperature == 293.0
    assert os.path.basename(m.config.plugin_path) == "libvpd_gpu.so"  # the stock JC on the GPU


def test_point_case_errors(tmp_path):
    with open(golden("examples/jc_material_point.json")) as f:
        case = json.load(f)
    case["materials"][0].update(materialConfigPath="configs/elastic.json", equivalentPlasticStrainIndex=0,
                                internalIndicator={"indices": [0]})
    p = tmp_path / "case.json"
    p.write_text(json.dumps(case))
    with pytest.raises(ValueError, match="plugin directory"):
        load_point_case(str(p), golden(""))
    with pytest.raises(RuntimeError, match="Failed to load VUMAT plugin"):
        run_material_point_case(str(p), str(tmp_path / "o"), golden(""), str(tmp_path),
                                log=lambda *a: None)
    case["materials"][0]["initialState"] = [0.0, 1.0]
    p.write_text(json.dumps(case))
    with pytest.raises(ValueError, match="initialState length"):
        load_point_case(str(p), golden(""), O.REF_DIR)
    case["materials"][0].pop("initialState")
    for edit, message in ((lambda d: d["time_integration"].update(steps=599), "totalTime"),
                          (lambda d: d["boundary_conditions"].update(mode="biaxial"), "type or mode"),
                          (lambda d: d.update(type="vumat_pd_boundary_case"), "vumat_material_point_case")):
        bad = json.loads(json.dumps(case))
        edit(bad)
        p.write_text(json.dumps(bad))
        with pytest.raises(ValueError, match=message):
            load_point_case(str(p), golden(""), O.REF_DIR)


# ---------------------------------------------------------------- affine demo cases
def test_demo_case_loading():
    from vpd.point_runner import load_affine_case
    case = load_affine_case(golden("examples/affine_shear_elastic.json"), "vumat_pd_demo_case",
                            golden(""), O.REF_DIR)
    assert (case.nx, case.ny, case.nz, case.spacing, case.horizon) == (5, 3, 3, 1.0, 1.75)
    assert (case.steps, case.mode, case.max_strain, case.damage_model) == (20, "simple_shear_xy", 1e-4, "none")
    assert (case.deformation_gradient_tolerance, case.reference_stress_tolerance,
            case.net_force_tolerance) == (1e-12, 0.002, 1e-7)
    assert case.checks and case.materials[0].config.nstatev == 1 and case.materials[0].reference
    assert os.path.basename(case.materials[0].config.plugin_path) == "elastic_vumat_plugin.so"


def test_demo_case_errors(tmp_path):
    from vpd.demo_runner import run_demo_case
    with open(golden("examples/affine_bar_elastic.json")) as f:
        case = json.load(f)
    case["boundary_conditions"]["maxStrain"] = 0.0
    p = tmp_path / "case.json"
    p.write_text(json.dumps(case))
    with pytest.raises(ValueError, match="requires maxStrain"):
        run_demo_case(str(p), str(tmp_path / "o"), golden(""), O.REF_DIR, log=lambda *a: None)
    with pytest.raises(ValueError, match="plugin directory"):
        run_demo_case(golden("examples/affine_bar_elastic.json"), str(tmp_path / "o"), golden(""),
                      log=lambda *a: None)


def test_runner_refuses_unknown_case_types(tmp_path, capsys):
    from vpd.runner import main
    p = tmp_path / "case.json"
    p.write_text(json.dumps({"name": "x", "type": "vumat_pd_demo"}))
    assert main([str(p)]) == 1
    assert "Unsupported case type" in capsys.readouterr().err


# the reference's tests/config_rejection_test.py cases, through this runner's command line
REJECTED_MATERIALS = [
    ({"kinematicsMode": "legacy_small_strain"}, "Unsupported kinematicsMode"),
    ({"internalIndicator": {"indices": [1], "reduction": "sum"}}, "reduction must be"),
    ({"internalIndicator": {"indices": [1], "transform": "unknown"}}, "transform must be"),
    ({"initialState": [0.0], "initialStateOverrides": {"5": 1.0}}, "initialState length"),
    ({"equivalentPlasticStrainIndex": -2}, "outside nstatev"),
    ({"internalIndicator": {"indices": [1.5]}}, "nonnegative integer"),
    ({"internalIndicator": {"indices": ["1"]}}, "nonnegative integer"),
    ({"initialStateOverrides": {"1junk": 1.0}}, "Invalid initialStateOverrides index"),
    ({"initialState": [0.0, "bad", 0.0, 0.0, 0.0, 0.0, 0.0]}, "Expected numeric entries"),
    ({"initialState": "not an array"}, "Expected numeric array"),
    ({"internalIndicator": {"indices": "1"}}, "Expected integer array"),
]
REJECTED_TIMES = [("steps", 1.5, "representable integer"), ("steps", 2147483648, "representable integer"),
                  ("dt", 0.0, "dt > 0"), ("dt", -1.0, "dt > 0"), ("dt", 1.0e308, "duration must be finite")]


@pytest.mark.parametrize("edit, message",
                         [((lambda c, e=e: c["materials"][0].update(e)), m) for e, m in REJECTED_MATERIALS]
                         + [((lambda c, f=f, v=v: c["time_integration"].update({f: v})), m)
                            for f, v, m in REJECTED_TIMES])
def test_reference_config_rejections(tmp_path, capsys, edit, message):
    from vpd.runner import main
    with open(golden("examples/jc_material_point.json")) as f:
        case = json.load(f)
    edit(case)
    out = tmp_path / "must_not_run"
    case["output"]["directory"] = str(out)
    p = tmp_path / "invalid.json"
    p.write_text(json.dumps(case))
    assert main([str(p), "--config-root", golden("")]) == 1
    assert message in capsys.readouterr().err
    assert not out.exists()


def test_runner_command_line_runs_material_point_cases(tmp_path):
    """``python -m vpd.runner`` dispatches on the case type: the material-point example through
    the command line writes the reference CLI's files."""
    from vpd.runner import main
    rc = main([golden("examples/jc_material_point.json"), "--config-root", golden(""),
               "--plugin-dir", O.REF_DIR, "--out", str(tmp_path)])
    assert rc == 0
    assert (tmp_path / "timeseries.csv").read_bytes() == fixture("jc_material_point", "timeseries.csv")
