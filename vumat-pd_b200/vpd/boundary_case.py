"""The reference's JSON boundary-value cases, read into ``Case`` objects.

``load_boundary_case(path)`` reads a ``vumat_pd_boundary_case`` file (the reference's
benchmarks/tensile3d/cases/*.json schema, parsed by src/config/DemoConfig.cpp:281-331 with the
defaults of include/DemoConfig.hpp:13-107) and the material config files it names
(src/config/MaterialConfigJson.cpp:63-101), and returns a ``BoundaryCase``: one ``Case`` per
material entry plus what the output files need (labels, output cadence, acceptance limits).

Only what the device increment implements is accepted; anything else raises ``ValueError``
naming the field:
  * boundary type ``regional_smooth_displacement`` (half-cosine displacement of the load band,
    BoundaryConditions.cpp:70-79), loading component x (support ``left``, load ``right``) or
    y (``bottom``/``top``), rigid-body suppression on;
  * the stock Johnson-Cook plugin as the device update, or any other VUMAT plugin through the
    host plugin path (found in the plugin directory); the corotational stress frame, the
    legacy_vumat_pd tensor convention, eqps at state variable 2 or none, an initial state
    (``initialState``, ``initialStateOverrides``) and the diagnostics' internal indicator;
  * damage ``none``, ``critical_stretch`` or the point modes ``eqps_threshold`` and
    ``max_principal_strain`` (with ``deletionEnabled``).
"""
from __future__ import annotations

import dataclasses
import json
import math
import os

import numpy as np

from .vumat_plugin import load_vumat_config
from .case import (BC_SMOOTH_DISPLACEMENT, DAMAGE_CRITICAL_STRETCH, DAMAGE_EQPS_THRESHOLD,
                   DAMAGE_MAX_PRINCIPAL_STRAIN, DAMAGE_NONE, Case)


@dataclasses.dataclass
class MaterialRun:
    """One material entry of a case: its ``Case`` and what its outputs report."""
    label: str
    case: Case
    elastic_e: float                 # for the analytical plane-strain slope E / (1 - nu^2)
    elastic_nu: float
    eqps_index: int                  # state variable written as eqps (-1: none)
    source_density: float            # the material config's density (kg/m^3)
    host_plugin: object = None       # VumatConfig of a plugin run on the host (None: device JC)
    initial_state: tuple = ()        # every point's starting VUMAT state (empty: zeros)
    indicator: tuple = None          # (indices, reduction, transform) of internalIndicator


@dataclasses.dataclass
class BoundaryCase:
    name: str
    classification: str
    scope: str
    steps: int
    dt: float
    output_every: int
    snapshot_every: int              # 0: only the last step
    component: str                   # "x" or "y"
    support_region: str
    load_region: str
    energy_tolerance: float
    net_force_tolerance: float
    minimum_plastic_strain: float
    kinetic_to_internal_limit: float
    output_directory: str
    materials: list


def _get(obj, key, default, kind):
    if key not in obj:
        return default
    value = obj[key]
    if kind is float:
        if isinstance(value, bool) or not isinstance(value, (int, float)):
            raise ValueError(f"{key} must be a number")
        return float(value)
    if kind is int:
        if isinstance(value, bool) or not isinstance(value, (int, float)) or int(value) != value:
            raise ValueError(f"{key} must be an integer")
        return int(value)
    if kind is bool:
        if not isinstance(value, bool):
            raise ValueError(f"{key} must be true or false")
        return value
    if not isinstance(value, str):
        raise ValueError(f"{key} must be a string")
    return value


def _section(root, key):
    obj = root.get(key, {})
    if not isinstance(obj, dict):
        raise ValueError(f"{key} must be a JSON object")
    return obj


def load_material_config(path: str, plugin_dir: str = None) -> dict:
    """A VUMAT material config (configs/*.json; MaterialConfigJson.cpp:63-101). The stock
    Johnson-Cook plugin runs as the device update; any other plugin (found as
    ``vpd.vumat_plugin.load_vumat_config`` finds it) runs through the host plugin path
    (``Simulation.set_host_vumat``), and its entry is returned as ``host_plugin``."""
    from . import library_path
    try:
        cfg = load_vumat_config(path, plugin_dir)
    except ValueError as e:
        raise ValueError(f"{path}: {e}") from None
    if cfg.stress_frame != "corotational":
        raise ValueError(f"{path}: boundary cases need the corotational stress frame")
    if cfg.plugin_path == library_path():  # the device Johnson-Cook update
        if cfg.cmname.upper() != "JOHNSONCOOK" or len(cfg.props) != 14 or cfg.nstatev != 6:
            raise ValueError(f"{path}: the Johnson-Cook plugin needs cmname JOHNSONCOOK, 14 props "
                             "and 6 state variables")
        return {"props": cfg.props, "nstatev": 6, "density": cfg.density, "host_plugin": None}
    if not cfg.props:
        raise ValueError(f"{path}: VUMAT props cannot be empty.")
    # the case's own 14 props are not read with a host plugin; the state keeps at least the 6
    # columns the device layout has
    return {"props": (0.0,) * 14, "nstatev": max(6, cfg.nstatev), "density": cfg.density,
            "host_plugin": cfg}


def _initial_state(entry: dict, label: str, nstatev: int) -> tuple:
    """initialState and initialStateOverrides of a material entry (DemoConfig.cpp:220-251), with
    the reference's checks and messages."""
    from .point_runner import _double_array
    state = _double_array(entry, "initialState")
    if state and len(state) != nstatev:
        raise ValueError("initialState length does not match nstatev.")
    overrides = entry.get("initialStateOverrides")
    if isinstance(overrides, dict):
        if not state:
            state = [0.0] * nstatev
        for key, value in overrides.items():
            if not key or not all("0" <= ch <= "9" for ch in key):
                raise ValueError("Invalid initialStateOverrides index for material: " + label)
            if not int(key) < nstatev or isinstance(value, bool) or not isinstance(value, (int, float)):
                raise ValueError("Invalid initialStateOverrides entry for material: " + label)
            state[int(key)] = float(value)
    return tuple(state)


def _indicator(entry: dict, label: str, nstatev: int):
    """internalIndicator of a material entry (DemoConfig.cpp:252-266), with the reference's checks."""
    from .point_runner import _int_array
    obj = entry.get("internalIndicator")
    if not isinstance(obj, dict):
        return None
    indices = _int_array(obj, "indices")
    reduction, transform = obj.get("reduction", "max"), obj.get("transform", "identity")
    if reduction not in ("min", "max"):
        raise ValueError("internalIndicator.reduction must be min or max.")
    if transform not in ("identity", "one_minus"):
        raise ValueError("internalIndicator.transform must be identity or one_minus.")
    if any(not 0 <= i < nstatev for i in indices):
        raise ValueError("internalIndicator index is outside nstatev for material: " + label)
    if len(indices) > 8:
        raise ValueError(f"material {label}: internalIndicator: at most 8 state variables on the device")
    return (tuple(indices), reduction, transform) if indices else None


def indicator_values(indicator, state: np.ndarray) -> np.ndarray:
    """Per point the internal indicator of the state rows (BoundaryValueCaseRunner.cpp:93-107):
    0 without one; else the min or max of the chosen variables (NaN skipped as std::min and
    std::max skip it), 1 minus that for one_minus."""
    if indicator is None:
        return np.zeros(state.shape[0])
    indices, reduction, transform = indicator
    value = np.full(state.shape[0], np.inf if reduction == "min" else -np.inf)
    for k in indices:
        item = state[:, k]
        value = np.where(item < value, item, value) if reduction == "min" else np.where(value < item, item, value)
    return 1.0 - value if transform == "one_minus" else value


def load_boundary_case(path: str, config_root: str = None, plugin_dir: str = None) -> BoundaryCase:
    """Reads a boundary-value case file. Material config paths are resolved against
    ``config_root`` (default: the current directory, as the reference's host resolves them),
    plugins other than the stock Johnson-Cook one against ``plugin_dir``."""
    with open(path) as f:
        root = json.load(f)
    if _get(root, "schemaVersion", "1.0", str) != "1.0":
        raise ValueError("unsupported case schemaVersion")
    name = _get(root, "name", None, str)
    if name is None:
        raise ValueError("the case needs a name")
    kind = _get(root, "type", "vumat_pd_demo", str)
    if kind != "vumat_pd_boundary_case":
        raise ValueError(f"type {kind!r}: only vumat_pd_boundary_case files run here")

    geo = _section(root, "geometry") or _section(root, "grid")
    if _get(geo, "type", "patch", str) != "patch":
        raise ValueError("geometry.type must be patch")
    nx, ny, nz = (_get(geo, k, 1, int) for k in ("nx", "ny", "nz"))
    spacing = _get(geo, "spacing", 1.0, float)
    horizon = _get(geo, "horizon", 1.0, float)

    ti = _section(root, "time_integration") or root
    steps = _get(ti, "steps", 1, int)
    dt = _get(ti, "dt", 1.0e-6, float)

    bc = _section(root, "boundary_conditions")
    bc_type = _get(bc, "type", "affine_displacement", str)
    if bc_type != "regional_smooth_displacement":
        raise ValueError(f"boundary_conditions.type {bc_type!r}: only regional_smooth_displacement runs here")
    component = _get(bc, "component", "x", str)
    support = _get(bc, "supportRegion", "left", str)
    load = _get(bc, "loadRegion", "right", str)
    expected = {"x": ("left", "right"), "y": ("bottom", "top")}
    if component not in expected:
        raise ValueError(f"boundary_conditions.component {component!r}: x or y")
    if (support, load) != expected[component]:
        raise ValueError(f"boundary_conditions: support {support!r} and load {load!r}: the device "
                         f"increment holds the {expected[component][0]} band and loads the "
                         f"{expected[component][1]} one")
    if not _get(bc, "rigidBodySuppression", False, bool):
        raise ValueError("boundary_conditions.rigidBodySuppression must be true: the device "
                         "increment always pins the rigid-body modes")
    region_layers = _get(bc, "regionLayers", 1, int)
    amplitude = _get(bc, "amplitude", 0.0, float)
    rise_time = _get(bc, "riseTime", 0.0, float)
    plane_strain = _get(bc, "planeStrain", False, bool)

    obs = _section(root, "observation")
    axial_min = _get(obs, "axialMin", math.nan, float)
    axial_max = _get(obs, "axialMax", math.nan, float)

    dyn = _section(root, "dynamics")
    density = _get(dyn, "density", 0.0, float)

    dmg = _section(root, "damage")
    model = _get(dmg, "model", "", str)
    modes = {"": DAMAGE_NONE, "none": DAMAGE_NONE, "critical_stretch": DAMAGE_CRITICAL_STRETCH,
             "Critical Stretch": DAMAGE_CRITICAL_STRETCH, "eqps_threshold": DAMAGE_EQPS_THRESHOLD,
             "max_principal_strain": DAMAGE_MAX_PRINCIPAL_STRAIN}
    if model not in modes:
        raise ValueError(f"damage.model {model!r}: none, critical_stretch, eqps_threshold or "
                         "max_principal_strain")
    damage_mode = modes[model]
    initiation = _get(dmg, "initiation", 0.0, float)
    if initiation <= 0.0:
        initiation = _get(dmg, "criticalStretch", initiation, float)
    failure = _get(dmg, "failure", 1.0, float)  # SimpleDamageConfig's default
    deletion = _get(dmg, "deletionEnabled", False, bool)

    out = _section(root, "output")
    materials = root.get("materials")
    if not isinstance(materials, list) or not materials:
        raise ValueError("the case needs a materials array")
    runs = []
    for entry in materials:
        if not isinstance(entry, dict):
            raise ValueError("each materials entry must be a JSON object")
        label = _get(entry, "name", None, str)
        if label is None:
            raise ValueError("each material needs a name")
        rel = _get(entry, "materialConfigPath", _get(entry, "configPath", _get(entry, "material_config_path", "", str), str), str)
        if not rel:
            raise ValueError(f"material {label}: materialConfigPath is required")
        if _get(entry, "kinematicsMode", "corotational", str) != "corotational":
            raise ValueError(f"material {label}: kinematicsMode must be corotational")
        cfg = load_material_config(os.path.join(config_root or ".", rel), plugin_dir)
        eqps_index = _get(entry, "equivalentPlasticStrainIndex", -1, int)
        nstatev = cfg["host_plugin"].nstatev if cfg["host_plugin"] else cfg["nstatev"]
        if not -1 <= eqps_index < nstatev:
            raise ValueError(f"material {label}: equivalentPlasticStrainIndex outside nstatev")
        if eqps_index not in (-1, 1):
            raise ValueError(f"material {label}: the device reduces state variable 2 as eqps; "
                             "equivalentPlasticStrainIndex must be 1 or -1")
        initial_state = _initial_state(entry, label, nstatev)
        indicator = _indicator(entry, label, nstatev)
        case = Case(name=f"{name}/{label}", nx=nx, ny=ny, nz=nz, spacing=spacing, horizon=horizon,
                    dt=dt, steps=steps, density=density, props=cfg["props"],
                    bc_mode=BC_SMOOTH_DISPLACEMENT, load_axis=0 if component == "x" else 1,
                    region_layers=region_layers, plane_strain=plane_strain, amplitude=amplitude,
                    rise_time=rise_time, observation_min=axial_min, observation_max=axial_max,
                    nstatev=cfg["nstatev"],
                    reference_temperature=_get(entry, "referenceTemperature", 293.0, float),
                    damage_mode=damage_mode, damage_initiation=initiation, damage_failure=failure,
                    damage_deletion=deletion)
        runs.append(MaterialRun(label=label, case=case, elastic_e=_get(entry, "elasticE", 0.0, float),
                                elastic_nu=_get(entry, "elasticNu", 0.0, float), eqps_index=eqps_index,
                                source_density=cfg["density"], host_plugin=cfg["host_plugin"],
                                initial_state=initial_state, indicator=indicator))
    return BoundaryCase(
        name=name, classification=_get(root, "classification", "verification", str),
        scope=_get(root, "scope", "", str), steps=steps, dt=dt,
        output_every=_get(dyn, "outputEvery", 1, int), snapshot_every=_get(dyn, "snapshotEvery", 0, int),
        component=component, support_region=support, load_region=load,
        energy_tolerance=_get(dyn, "energyToleranceRelative", 1.0e-3, float),
        net_force_tolerance=_get(dyn, "netForceTolerance", 1.0e-8, float),
        minimum_plastic_strain=_get(dyn, "minimumPlasticStrain", 0.0, float),
        kinetic_to_internal_limit=_get(dyn, "kineticToInternalLimit", 1.0, float),
        output_directory=_get(out, "directory", "validation_cases/output/" + name, str),
        materials=runs)
