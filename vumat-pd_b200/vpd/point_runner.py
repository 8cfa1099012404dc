"""The reference's material-point case (``"type": "vumat_material_point_case"``, e.g. its
examples/jc_material_point.json, the README's quick start): one material point driven through
a prescribed strain path by a VUMAT plugin, written as the reference's ``timeseries.csv`` and
``metadata.json``.

The case is MaterialPointCaseRunner.cpp:73-234: every step loads the point to
``maxStrain * step / steps`` in the case's mode (``uniaxial_xx``, ``simple_shear_xy``, or
``plane_strain_x_uniaxial_stress``, where a bisection on the lateral strain drives the lateral
stress to zero, :116-150), and each evaluation is one ``vumat_adapter_call`` of the material's
plugin (``vpd.vumat_plugin``). The stock Johnson-Cook plugin is this package's library, so the
routine runs on the GPU; the steps are serial, one plugin call per evaluation.

Output text matches the reference's: the stream's 16 significant digits in both files, the
same columns, keys and order.
"""
from __future__ import annotations

import dataclasses
import json
import math
import os

import numpy as np

from .vumat_plugin import PointInput, PointResult, VumatPlugin, load_vumat_config

TIMESERIES_HEADER = ("material,step,time,applied_strain,stress,elastic_reference_stress,"
                     "reference_error,state_indicator,internal_energy,inelastic_energy,"
                     "temperature,lateral_strain,finite\n")


def g16(x: float) -> str:
    return "%.16g" % x


@dataclasses.dataclass
class PointMaterial:
    label: str
    config: object                   # VumatConfig
    reference: bool
    elastic_e: float
    elastic_nu: float
    reference_temperature: float
    initial_state: list
    indicator_indices: list
    indicator_reduction: str
    indicator_transform: str


@dataclasses.dataclass
class AffineCase:
    """A material-point or affine demo case: the fields of DemoCaseConfig these hosts read."""
    name: str
    scope: str
    nx: int
    ny: int
    nz: int
    spacing: float
    horizon: float
    steps: int
    dt: float
    mode: str
    max_strain: float
    reference_stress_tolerance: float
    deformation_gradient_tolerance: float
    net_force_tolerance: float
    damage_model: str            # SimpleDamageConfig::mode
    damage_initiation: float
    damage_failure: float
    damage_deletion: bool
    checks: list
    output_directory: str
    materials: list


def _num(obj, key, default):
    """getDouble (SimpleJson.cpp:281-291)."""
    value = obj.get(key, default)
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise ValueError("Expected numeric field: " + key)
    return value


def _int(obj, key, default):
    """getInt (SimpleJson.cpp:264-279): a number with an exact 32-bit integer value."""
    value = _num(obj, key, default)
    if not math.isfinite(value) or math.trunc(value) != value or not -2**31 <= value <= 2**31 - 1:
        raise ValueError("Expected representable integer field: " + key)
    return int(value)


def _double_array(obj, key):
    """loadOptionalDoubleArray (DemoConfig.cpp:173-187)."""
    if key not in obj:
        return []
    value = obj[key]
    if not isinstance(value, list):
        raise ValueError("Expected numeric array: " + key)
    if any(isinstance(v, bool) or not isinstance(v, (int, float)) for v in value):
        raise ValueError("Expected numeric entries in " + key)
    return [float(v) for v in value]


def _int_array(obj, key):
    """loadOptionalIntArray (DemoConfig.cpp:189-204): non-negative integers."""
    if key not in obj:
        return []
    value = obj[key]
    if not isinstance(value, list):
        raise ValueError("Expected integer array: " + key)
    out = []
    for v in value:
        if isinstance(v, bool) or not isinstance(v, (int, float)) or not math.isfinite(v) \
                or math.trunc(v) != v or v < 0 or v > 2**31 - 1:
            raise ValueError("Expected nonnegative integer entries in " + key)
        out.append(int(v))
    return out


def _load_material(entry, config_root, plugin_dir) -> PointMaterial:
    """loadMaterial, DemoConfig.cpp:206-268."""
    label = entry.get("name")
    if not isinstance(label, str):
        raise ValueError("each material needs a name")
    rel = entry.get("materialConfigPath", entry.get("configPath", entry.get("material_config_path", "")))
    if not rel:
        raise ValueError("Material entry requires materialConfigPath or configPath.")
    config = load_vumat_config(os.path.join(config_root or ".", rel), plugin_dir)
    if config.stress_frame != "corotational":
        raise ValueError("JSON case hosts require corotational stress; use the dedicated spatial demo.")
    if entry.get("kinematicsMode", "corotational") != "corotational":
        raise ValueError("Unsupported kinematicsMode for material: " + label)
    state = _double_array(entry, "initialState")
    if state and len(state) != config.nstatev:
        raise ValueError("initialState length does not match nstatev.")
    eqps = _int(entry, "equivalentPlasticStrainIndex", -1)
    if not -1 <= eqps < config.nstatev:
        raise ValueError("equivalentPlasticStrainIndex is outside nstatev for material: " + label)
    overrides = entry.get("initialStateOverrides")
    if isinstance(overrides, dict):
        if not state:
            state = [0.0] * config.nstatev
        for key, value in overrides.items():
            if not key or not all("0" <= ch <= "9" for ch in key):
                raise ValueError("Invalid initialStateOverrides index for material: " + label)
            if not int(key) < config.nstatev or isinstance(value, bool) or not isinstance(value, (int, float)):
                raise ValueError("Invalid initialStateOverrides entry for material: " + label)
            state[int(key)] = float(value)
    if state and len(state) != config.nstatev:
        raise ValueError("initialState length does not match nstatev for material: " + label)
    indices, reduction, transform = [], "max", "identity"
    indicator = entry.get("internalIndicator")
    if isinstance(indicator, dict):
        indices = _int_array(indicator, "indices")
        reduction = indicator.get("reduction", "max")
        transform = indicator.get("transform", "identity")
        if reduction not in ("min", "max"):
            raise ValueError("internalIndicator.reduction must be min or max.")
        if transform not in ("identity", "one_minus"):
            raise ValueError("internalIndicator.transform must be identity or one_minus.")
        if any(not 0 <= i < config.nstatev for i in indices):
            raise ValueError("internalIndicator index is outside nstatev for material: " + label)
    return PointMaterial(label=label, config=config, reference=bool(entry.get("reference", False)),
                         elastic_e=float(_num(entry, "elasticE", 0.0)),
                         elastic_nu=float(_num(entry, "elasticNu", 0.0)),
                         reference_temperature=float(_num(entry, "referenceTemperature", 293.0)),
                         initial_state=state, indicator_indices=indices,
                         indicator_reduction=reduction, indicator_transform=transform)


def load_point_case(path: str, config_root: str | None = None, plugin_dir: str | None = None) -> AffineCase:
    """A ``vumat_material_point_case`` file."""
    return load_affine_case(path, "vumat_material_point_case", config_root, plugin_dir)


def load_affine_case(path: str, kind: str, config_root: str | None = None,
                     plugin_dir: str | None = None) -> AffineCase:
    """A ``vumat_material_point_case`` or ``vumat_pd_demo_case`` file (loadDemoCaseConfigFromJson,
    DemoConfig.cpp:285-354, with its defaults and checks)."""
    with open(path) as f:
        root = json.load(f)
    if root.get("schemaVersion", "1.0") != "1.0":
        raise ValueError("Unsupported VUMAT-PD case schemaVersion: " + str(root.get("schemaVersion")))
    if root.get("type", "vumat_pd_demo") != kind:
        raise ValueError(f"not a {kind} file")
    name = root.get("name")
    if not isinstance(name, str):
        raise ValueError("the case needs a name")
    geo = root.get("geometry") if isinstance(root.get("geometry"), dict) else root.get("grid", {})
    ti = root.get("time_integration") if isinstance(root.get("time_integration"), dict) else root
    bc = root.get("boundary_conditions") if isinstance(root.get("boundary_conditions"), dict) else None
    mode = bc.get("mode", "uniaxial_xx") if bc is not None else "uniaxial_xx"
    bc_type = bc.get("type", "affine_displacement") if bc is not None else "affine_displacement"
    max_strain = _num(bc if bc is not None else root, "maxStrain", 0.0)
    # the loader's checks (DemoConfig.cpp:332-354)
    if not (_num(geo, "spacing", 1.0) > 0.0 and _num(geo, "horizon", 1.0) > 0.0):
        raise ValueError("PD geometry requires positive spacing and horizon.")
    if geo.get("type", "patch") != "patch":
        raise ValueError("Unsupported geometry type: " + str(geo.get("type")))
    if min(_int(geo, k, 1) for k in ("nx", "ny", "nz")) < 2:
        raise ValueError("PD patch geometry requires nx/ny/nz >= 2.")
    steps, dt = _int(ti, "steps", 1), float(_num(ti, "dt", 1.0e-6))
    if steps < 1 or not math.isfinite(dt) or dt <= 0.0:
        raise ValueError("time_integration requires steps >= 1 and dt > 0.")
    total = float(_num(ti, "totalTime", 0.0))
    expected = dt * steps
    if total <= 0.0:
        total = expected
    if not math.isfinite(expected) or not math.isfinite(total):
        raise ValueError("time_integration duration must be finite.")
    if abs(total - expected) > 1.0e-12 * max(1.0, expected):
        raise ValueError("time_integration.totalTime must equal steps * dt.")
    if bc_type != "affine_displacement" or mode not in (
            "uniaxial_xx", "simple_shear_xy", "plane_strain_x_uniaxial_stress"):
        raise ValueError("Unsupported boundary_conditions type or mode.")
    tol = root.get("tolerances") if isinstance(root.get("tolerances"), dict) else {}
    out = root.get("output") if isinstance(root.get("output"), dict) else {}
    dmg = root.get("damage") if isinstance(root.get("damage"), dict) else {}  # loadDamage, :117-134
    model = dmg.get("model", "")
    model = "critical_stretch" if model in ("critical_stretch", "Critical Stretch") else (model or "none")
    initiation = float(_num(dmg, "initiation", 0.0))
    if initiation <= 0.0:
        initiation = float(_num(dmg, "criticalStretch", initiation))
    checks = [c for c in root.get("checks", []) if isinstance(c, str)] if isinstance(root.get("checks"), list) else []
    materials = root.get("materials")
    if not isinstance(materials, list):
        raise ValueError("Demo case requires a materials array.")
    runs = []
    for entry in materials:
        if not isinstance(entry, dict):
            raise ValueError("Each materials entry must be a JSON object.")
        runs.append(_load_material(entry, config_root, plugin_dir))
    if not runs:
        raise ValueError("Demo case requires at least one material.")
    return AffineCase(name=name, scope=root.get("scope", ""), nx=_int(geo, "nx", 1),
                      ny=_int(geo, "ny", 1), nz=_int(geo, "nz", 1),
                      spacing=float(_num(geo, "spacing", 1.0)), horizon=float(_num(geo, "horizon", 1.0)),
                      steps=steps, dt=dt, mode=mode, max_strain=float(max_strain),
                      reference_stress_tolerance=float(_num(tol, "referenceStressAbsolute", 1.0e-6)),
                      deformation_gradient_tolerance=float(_num(tol, "deformationGradientAbsolute", 1.0e-12)),
                      net_force_tolerance=float(_num(tol, "netForceAbsolute", 1.0e-7)),
                      damage_model=model, damage_initiation=initiation,
                      damage_failure=float(_num(dmg, "failure", 1.0)),
                      damage_deletion=bool(dmg.get("deletionEnabled", False)), checks=checks,
                      output_directory=out.get("directory", "validation_cases/output/" + name),
                      materials=runs)


def reference_stress(m: PointMaterial, load: float, mode: str) -> float:
    """Elastic reference stress of the loading mode (:32-44)."""
    e, nu = m.elastic_e, m.elastic_nu
    if e <= 0.0:
        return 0.0
    mu = e / (2.0 * (1.0 + nu))
    if mode == "simple_shear_xy":
        return mu * load
    if mode == "plane_strain_x_uniaxial_stress":
        return e / (1.0 - nu * nu) * load
    lam = e * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return (lam + 2.0 * mu) * load


def state_indicator(m: PointMaterial, state) -> float:
    """The internal indicator of a state vector (:46-59)."""
    if not m.indicator_indices:
        return 0.0
    value = math.inf if m.indicator_reduction == "min" else -math.inf
    for k in m.indicator_indices:
        c = state[k]
        if m.indicator_reduction == "min":
            value = c if c < value else value
        else:
            value = c if value < c else value
    if m.indicator_transform == "one_minus":
        value = 1.0 - value
    return value if 0.0 < value else 0.0


def _finite(values) -> bool:
    return all(math.isfinite(v) for v in values)


def _trials(plugin: VumatPlugin, inp: PointInput, previous_lateral: float, laterals) -> list:
    """The plugin on one row per trial lateral strain (the evaluate lambda of :117-125), all
    rows in one block call; each row is computed independently of the others."""
    rows = len(laterals)

    def tile(values):
        return np.tile(np.asarray(values, dtype=np.float64), (rows, 1))

    lat = np.asarray(laterals, dtype=np.float64)
    strain_rate, strain_n = tile(inp.strain_rate), tile(inp.strain_n)
    defgrad_old, defgrad_new = tile(inp.defgrad_old), tile(inp.defgrad_new)
    strain_rate[:, 4] = (lat - previous_lateral) / inp.dt
    strain_n[:, 4] = previous_lateral
    defgrad_old[:, 4] = 1.0 + previous_lateral
    defgrad_new[:, 4] = 1.0 + lat
    r = plugin.update_block(dt=inp.dt, step_time=inp.step_time, total_time=inp.total_time,
                            char_length=np.full(rows, inp.char_length),
                            temperature=np.full(rows, inp.temperature), strain_rate=strain_rate,
                            rel_spin=tile(inp.rel_spin), stress_n=tile(inp.stress_n),
                            stretch_old=tile(inp.stretch_old), stretch_new=tile(inp.stretch_new),
                            defgrad_old=defgrad_old, defgrad_new=defgrad_new,
                            state_old=tile(inp.state_old).reshape(rows, -1),
                            internal_energy_old=np.full(rows, inp.internal_energy_old),
                            inelastic_energy_old=np.full(rows, inp.inelastic_energy_old))
    return [PointResult(stress=r["stress"][k].tolist(), state=r["state"][k].tolist(),
                        temperature=float(r["temperature"][k]),
                        internal_energy=float(r["internal_energy"][k]),
                        inelastic_energy=float(r["inelastic_energy"][k])) for k in range(rows)]


# levels of the bisection tree per plugin call: 8 (255 rows in one block) when the plugin is
# this package's library, whose rows run in parallel on the GPU and whose cost is the round
# trip; 1 for a host plugin, which would compute every speculative row
TREE_LEVELS_DEVICE = 8


def _plane_strain_bisection(plugin: VumatPlugin, inp: PointInput, load: float, previous_lateral: float,
                            tree_levels: int):
    """The reference's bisection on the lateral strain for zero lateral stress (:126-150),
    evaluated ``tree_levels`` levels at a time. The interval of every node of the bisection tree
    follows from the path alone (midpoint 0.5 (lower + upper), left keeps lower, right keeps
    upper), so the next levels' midpoints go to the plugin as one block; the walk down the
    tree then takes the reference's branch at each node from the residuals. It visits the
    reference's midpoints with the same values and stops where it stops, so the lateral
    strain and the result are the reference's; the other nodes' rows are discarded."""
    lower, upper = -load, 0.25 * load
    if tree_levels == 1:  # one midpoint per call, as the reference runs it
        def evaluate(trial_lateral):
            trial = inp.copy()
            trial.strain_rate[4] = (trial_lateral - previous_lateral) / inp.dt
            trial.strain_n[4] = previous_lateral
            trial.defgrad_old[4] = 1.0 + previous_lateral
            trial.defgrad_new[4] = 1.0 + trial_lateral
            return plugin.update_point(trial)

        lower_residual = evaluate(lower).stress[4]
        upper_residual = evaluate(upper).stress[4]
        if lower_residual * upper_residual > 0.0:
            raise RuntimeError("Could not bracket zero lateral stress in material-point reference.")
        lateral, result = 0.0, None
        for _ in range(36):
            lateral = 0.5 * (lower + upper)
            result = evaluate(lateral)
            residual = result.stress[4]
            if abs(residual) < 1.0e-8:
                break
            if lower_residual * residual <= 0.0:
                upper, upper_residual = lateral, residual
            else:
                lower, lower_residual = lateral, residual
        return lateral, result
    bracket = _trials(plugin, inp, previous_lateral, [lower, upper])
    lower_residual, upper_residual = bracket[0].stress[4], bracket[1].stress[4]
    if lower_residual * upper_residual > 0.0:
        raise RuntimeError("Could not bracket zero lateral stress in material-point reference.")
    lateral, result, iteration = 0.0, None, 0
    while iteration < 36:
        levels = min(tree_levels, 36 - iteration)
        nodes = [(lower, upper)]  # heap order: node k has children 2k+1 (left) and 2k+2 (right)
        mids = []
        for k in range((1 << levels) - 1):
            lo, up = nodes[k]
            mid = 0.5 * (lo + up)
            mids.append(mid)
            if 2 * k + 2 < (1 << levels) - 1:
                nodes.append((lo, mid))
                nodes.append((mid, up))
        results = _trials(plugin, inp, previous_lateral, mids)
        k = 0
        for _ in range(levels):
            lateral, result = mids[k], results[k]
            residual = result.stress[4]
            iteration += 1
            if abs(residual) < 1.0e-8:
                return lateral, result
            if lower_residual * residual <= 0.0:
                upper, upper_residual = lateral, residual
                k = 2 * k + 1
            else:
                lower, lower_residual = lateral, residual
                k = 2 * k + 2
    return lateral, result


def run_material(case: AffineCase, m: PointMaterial, lines: list, tree_levels: int | None = None) -> dict:
    """runMaterial (:73-183) for one material; appends its timeseries lines. ``tree_levels``
    (default: by the plugin, see TREE_LEVELS_DEVICE) sets the bisection levels per call."""
    from . import library_path
    plugin = VumatPlugin(m.config)
    if tree_levels is None:
        tree_levels = TREE_LEVELS_DEVICE if m.config.plugin_path == library_path() else 1
    if not 1 <= tree_levels <= 8:
        raise ValueError("tree_levels must be in [1, 8]")
    dt = case.dt
    inp = PointInput(dt=dt, char_length=case.spacing, temperature=m.reference_temperature,
                     state_old=list(m.initial_state) if m.initial_state else [0.0] * m.config.nstatev)
    summary = dict(name=m.label, reference=m.reference, finite=True, maxReferenceError=0.0,
                   finalStress=0.0, finalIndicator=0.0, finalInternalEnergy=0.0,
                   finalInelasticEnergy=0.0)
    previous_lateral = 0.0
    steps = case.steps
    for step in range(1, steps + 1):
        previous_load = case.max_strain * float(step - 1) / float(steps)
        load = case.max_strain * float(step) / float(steps)
        rate = (load - previous_load) / dt
        inp.step_time = float(step - 1) * dt
        inp.total_time = inp.step_time
        inp.strain_rate = [0.0] * 9
        inp.strain_n = [0.0] * 9
        inp.defgrad_old = [1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0]
        inp.defgrad_new = list(inp.defgrad_old)
        if case.mode == "simple_shear_xy":
            inp.strain_rate[1] = inp.strain_rate[3] = 0.5 * rate
            inp.strain_n[1] = inp.strain_n[3] = 0.5 * previous_load
            inp.defgrad_old[1] = previous_load
            inp.defgrad_new[1] = load
        else:
            inp.strain_rate[0] = rate
            inp.strain_n[0] = previous_load
            inp.defgrad_old[0] = 1.0 + previous_load
            inp.defgrad_new[0] = 1.0 + load
        lateral = 0.0
        if case.mode == "plane_strain_x_uniaxial_stress":
            lateral, result = _plane_strain_bisection(plugin, inp, load, previous_lateral, tree_levels)
            previous_lateral = lateral
        else:
            result = plugin.update_point(inp)
        s = result.stress
        stress = 0.5 * (s[1] + s[3]) if case.mode == "simple_shear_xy" else s[0]
        reference = reference_stress(m, load, case.mode)
        error = abs(stress - reference)
        indicator = state_indicator(m, result.state)
        finite = (_finite(s) and _finite(result.state) and math.isfinite(result.temperature)
                  and math.isfinite(result.internal_energy) and math.isfinite(result.inelastic_energy)
                  and math.isfinite(indicator))
        summary["finite"] = summary["finite"] and finite
        if m.reference and summary["maxReferenceError"] < error:
            summary["maxReferenceError"] = error
        summary.update(finalStress=stress, finalIndicator=indicator,
                       finalInternalEnergy=result.internal_energy,
                       finalInelasticEnergy=result.inelastic_energy)
        lines.append(",".join([m.label, str(step), g16(step * dt), g16(load), g16(stress), g16(reference),
                               g16(error), g16(indicator), g16(result.internal_energy),
                               g16(result.inelastic_energy), g16(result.temperature), g16(lateral),
                               "1" if finite else "0"]) + "\n")
        inp.stress_n = list(s)
        inp.state_old = list(result.state)
        inp.temperature = result.temperature
        inp.internal_energy_old = result.internal_energy
        inp.inelastic_energy_old = result.inelastic_energy
    return summary


def metadata_text(case: AffineCase, summaries: list, passed: bool) -> str:
    """metadata.json of runMaterialPointCase (:200-222)."""
    def b(v):
        return "true" if v else "false"

    items = [(f"    {{\"name\": \"{s['name']}\", \"reference\": {b(s['reference'])}, "
              f"\"finite\": {b(s['finite'])}, \"maxReferenceError\": {g16(s['maxReferenceError'])}, "
              f"\"finalStress\": {g16(s['finalStress'])}, \"finalIndicator\": {g16(s['finalIndicator'])}, "
              f"\"finalInternalEnergy\": {g16(s['finalInternalEnergy'])}, "
              f"\"finalInelasticEnergy\": {g16(s['finalInelasticEnergy'])}}}") for s in summaries]
    return (f"{{\n  \"name\": \"{case.name}\",\n  \"status\": \"{'pass' if passed else 'fail'}\",\n"
            f"  \"scope\": \"{case.scope}\",\n  \"steps\": {case.steps},\n  \"mode\": \"{case.mode}\",\n"
            "  \"materials\": [\n" + "".join(item + (",\n" if k + 1 < len(items) else "\n")
                                           for k, item in enumerate(items)) + "  ]\n}\n")


def run_material_point_case(path: str, out_dir: str | None = None, config_root: str | None = None,
                            plugin_dir: str | None = None, log=print, tree_levels: int | None = None) -> int:
    """Runs the case and writes its files; 0 when it passes, 2 when it does not (:185-234)."""
    case = load_point_case(path, config_root, plugin_dir)
    out = out_dir or case.output_directory
    os.makedirs(out, exist_ok=True)
    lines = [TIMESERIES_HEADER]
    summaries = [run_material(case, m, lines, tree_levels) for m in case.materials]
    passed = True
    for s in summaries:
        passed = passed and s["finite"]
        if s["reference"]:
            passed = passed and s["maxReferenceError"] < case.reference_stress_tolerance
    with open(os.path.join(out, "timeseries.csv"), "w") as f:
        f.write("".join(lines))
    with open(os.path.join(out, "metadata.json"), "w") as f:
        f.write(metadata_text(case, summaries, passed))
    for s in summaries:
        log(f"{s['name']}: final_stress={s['finalStress']:g} max_reference_error={s['maxReferenceError']:g} "
            f"state_indicator={s['finalIndicator']:g} finite={'true' if s['finite'] else 'false'}")
    log(f"Material-point case written to {out}")
    return 0 if passed else 2
