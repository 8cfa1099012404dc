"""Runs one of the reference's JSON case files (``python -m vpd.runner CASE.json``), as its
``vumat_pd_run`` does: by the case's ``type``, a boundary-value case (this module), a
material-point case (``vpd.point_runner``) or an affine demo case (``vpd.demo_runner``).

A boundary-value case runs on the GPU and writes the reference's output files: timeseries.csv, field_snapshots.csv and metadata.json in the layout of its case
runner (runBoundaryValueCase, src/host/BoundaryValueCaseRunner.cpp:341-439), so the
reference's analysis scripts read them unchanged.

    python -m vpd.runner benchmarks/tensile3d/cases/pd_coarse.json [--out DIR] [--config-root DIR]

Layout kept from the reference, because downstream tools parse it:
  * timeseries.csv: one row at step 1, every ``outputEvery`` steps and the last step; the
    material label, the step, then the diagnostics at 16 significant digits and the finite
    flag (BoundaryValueCaseRunner.cpp:300-309);
  * field_snapshots.csv: every point at every ``snapshotEvery`` step and the last one, at 16
    significant digits (:115-137);
  * metadata.json: the case description and, per material, the run summary that the reference
    accumulates over every increment (:281-297), numbers at 15 significant digits where the
    reference formats them that way and 6 where it uses the stream default (:367-438).
The increments themselves run through ``vpd.Simulation`` (the library's ``vpd_step``); the
device Johnson-Cook update stands in for the material config's plugin, and metadata names the
library that ran (``plugin_file``: libvpd_gpu.so).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np

from .boundary_case import BoundaryCase, indicator_values, load_boundary_case
from .case import DIAG

TIMESERIES_HEADER = (
    "material,step,time_ms,load_displacement_mm,load_velocity_mm_per_ms,reaction_force_N,"
    "engineering_strain,lateral_strain,nominal_stress_MPa,average_axial_strain,"
    "average_axial_stress_MPa,max_eqps,max_internal_indicator,kinetic_energy_Nmm,"
    "internal_energy_Nmm,external_work_Nmm,relative_energy_error,net_internal_force_N,finite\n")
SNAPSHOT_HEADER = (
    "material,step,time_ms,particle,x0_mm,y0_mm,z0_mm,ux_mm,uy_mm,uz_mm,x_mm,y_mm,z_mm,"
    "vx_mm_per_ms,vy_mm_per_ms,vz_mm_per_ms,axial_strain,axial_stress_MPa,eqps,"
    "internal_indicator,simple_damage\n")
# the diagnostics columns of a timeseries row, after the label and the step
_SERIES = ("time_ms", "load_displacement_mm", "load_velocity_mm_per_ms", "reaction_force_N",
           "engineering_strain", "lateral_strain", "nominal_stress_MPa", "average_axial_strain",
           "average_axial_stress_MPa", "max_eqps", "max_internal_indicator", "kinetic_energy_Nmm",
           "internal_energy_Nmm", "external_work_Nmm", "relative_energy_error", "net_internal_force_N")


def g16(x: float) -> str:
    """A double as a C++ stream with precision 16 prints it (%.16g)."""
    return "%.16g" % x


def g6(x: float) -> str:
    """A double at the stream's default precision (%.6g)."""
    return "%.6g" % x


def json_number(x: float) -> str:
    """The reference's jsonNumber: 15 significant digits, null when not finite."""
    return "%.15g" % x if math.isfinite(x) else "null"


def timeseries_line(label: str, row) -> str:
    """One timeseries.csv line from a diagnostics row (``vpd.DIAG`` columns)."""
    return (f"{label},{int(row[DIAG['step']])}," + ",".join(g16(row[DIAG[c]]) for c in _SERIES)
            + f",{1 if row[DIAG['finite']] != 0.0 else 0}\n")


def snapshot_lines(label: str, step: int, time_ms: float, x0, u, v, strain_axial, stress_axial,
                   eqps, damage, indicator=None) -> str:
    """field_snapshots.csv lines of every point at one step (``indicator``: the internal
    indicator per point, 0 when the material configures none)."""
    out = []
    t = g16(time_ms)
    for i in range(len(x0)):
        x = x0[i] + u[i]
        out.append(",".join([label, str(step), t, str(i)] + [g16(a) for a in x0[i]] + [g16(a) for a in u[i]]
                            + [g16(a) for a in x] + [g16(a) for a in v[i]]
                            + [g16(strain_axial[i]), g16(stress_axial[i]), g16(eqps[i]),
                               "0" if indicator is None else g16(indicator[i]), g16(damage[i])]) + "\n")
    return "".join(out)


def observation_bounds(positions: np.ndarray, axis: int, band: float, lo_req: float, hi_req: float):
    """The observation window along the loading axis: the requested bounds, or the inner edges
    of the two end bands where a bound is not given (include/ObservationWindow.hpp:13-29)."""
    lo, hi = float(positions[:, axis].min()), float(positions[:, axis].max())
    a = lo + band if math.isnan(lo_req) else lo_req
    b = hi - band if math.isnan(hi_req) else hi_req
    if not (math.isfinite(a) and math.isfinite(b)) or a < lo or b > hi or a >= b:
        raise ValueError("Observation window must lie within the body and have positive length.")
    return a, b


def summarise(rows: np.ndarray, elastic_e: float, elastic_nu: float) -> dict:
    """The run summary the reference accumulates over every increment, from all rows."""
    col = {k: rows[:, DIAG[k]] for k in DIAG}
    kinetic, internal = col["kinetic_energy_Nmm"], col["internal_energy_Nmm"]
    ratio = kinetic / np.maximum(np.abs(internal), 1.0e-12)
    x2 = xy = 0.0
    for e, s in zip(col["engineering_strain"], col["average_axial_stress_MPa"]):
        if 1.0e-6 < e <= 1.0e-3:  # in increment order, as the reference sums
            x2 += e * e
            xy += e * s
    slope = xy / x2 if x2 > 0.0 else 0.0
    analytical = elastic_e / (1.0 - elastic_nu * elastic_nu)
    return {
        "maxNetInternalForce": float(col["net_internal_force_N"].max()),
        "finalEnergyError": float(col["relative_energy_error"][-1]),
        "maxEnergyError": float(col["relative_energy_error"].max()),
        "maxKineticToInternal": float(ratio.max()), "finalKineticToInternal": float(ratio[-1]),
        "maxEqps": float(col["max_eqps"].max()), "maxInternalIndicator": float(col["max_internal_indicator"].max()),
        "earlyElasticSlope": slope, "analyticalPlaneStrainSlope": analytical,
        "earlyElasticRelativeError": abs(slope - analytical) / analytical if analytical > 0.0 else 0.0,
        "finalReaction": float(col["reaction_force_N"][-1]),
        "finalNominalStress": float(col["nominal_stress_MPa"][-1]),
        "finalEngineeringStrain": float(col["engineering_strain"][-1]),
        "finite": bool(np.all(col["finite"] != 0.0)),
    }


def passes(bc: BoundaryCase, s: dict) -> bool:
    return (s["finite"] and s["maxNetInternalForce"] <= bc.net_force_tolerance
            and s["finalEnergyError"] <= bc.energy_tolerance
            and s["finalKineticToInternal"] <= bc.kinetic_to_internal_limit
            and s["maxEqps"] >= bc.minimum_plastic_strain)


def metadata_text(bc: BoundaryCase, summaries: list) -> str:
    """metadata.json in the reference's layout; ``summaries`` holds one dict per material with
    the summarise() fields plus label, pass, runtimeSeconds, observationMin, observationMax."""
    c = bc.materials[0].case
    ok = all(s["pass"] for s in summaries)
    head = (
        "{\n"
        f"  \"name\": \"{bc.name}\",\n"
        "  \"solver\": \"correspondence peridynamics\",\n"
        f"  \"status\": \"{'pass' if ok else 'fail'}\",\n"
        f"  \"classification\": \"{bc.classification}\",\n"
        f"  \"scope\": \"{bc.scope}\",\n"
        "  \"units\": {\"length\": \"mm\", \"time\": \"ms\", \"force\": \"N\", \"stress\": \"MPa\", "
        "\"solverMassDensity\": \"N*ms^2/mm^4\", \"sourceDensity\": \"kg/m^3\"},\n"
        "  \"densityConversion\": \"rho_solver = rho_kg_per_m3 * 1e-6\",\n"
        f"  \"particles\": {c.nx * c.ny * c.nz},\n"
        f"  \"grid\": [{c.nx},{c.ny},{c.nz}],\n  \"spacing_mm\": {g6(c.spacing)},\n"
        f"  \"horizon_mm\": {g6(c.horizon)},\n  \"horizonSpacingRatio\": {g6(c.horizon / c.spacing)},\n"
        "  \"neighborSearch\": \"cell-linked-list\",\n"
        f"  \"planeStrain\": {'true' if c.plane_strain else 'false'},\n"
        f"  \"outerSimpleDamage\": {'true' if c.damage_mode else 'false'},\n"
        "  \"zeroEnergyStabilization\": \"none\",\n"
        "  \"timeStepPolicy\": \"user supplied; no computed stability bound\",\n"
        f"  \"boundarySets\": {{\"support\": \"{bc.support_region}\", \"loaded\": \"{bc.load_region}\", "
        f"\"regionLayers\": {c.region_layers}, \"rigidBodySuppression\": \"two lateral components at "
        "support centre and z at support upper midplane point\"},\n"
        f"  \"dt_ms\": {g6(bc.dt)},\n  \"steps\": {bc.steps},\n  \"materials\": [\n")
    items = []
    for m, s in zip(bc.materials, summaries):
        items.append(
            f"    {{\"name\": \"{m.label}\", \"status\": \"{'pass' if s['pass'] else 'fail'}\", "
            f"\"plugin_file\": \"{plugin_file(m)}\", \"sourceDensity_kg_per_m3\": {json_number(m.source_density)}, "
            f"\"solverDensity\": {json_number(m.case.density)}, \"runtimeSeconds\": {json_number(s['runtimeSeconds'])}, "
            f"\"observationAxis\": \"{bc.component}\", \"observationMin_mm\": {json_number(s['observationMin'])}, "
            f"\"observationMax_mm\": {json_number(s['observationMax'])}, "
            f"\"maxNetInternalForce_N\": {json_number(s['maxNetInternalForce'])}, "
            f"\"finalEnergyError\": {json_number(s['finalEnergyError'])}, "
            f"\"maxEnergyError\": {json_number(s['maxEnergyError'])}, "
            f"\"maxKineticToInternal\": {json_number(s['maxKineticToInternal'])}, "
            f"\"finalKineticToInternal\": {json_number(s['finalKineticToInternal'])}, "
            f"\"maxEqps\": {json_number(s['maxEqps'])}, \"maxInternalIndicator\": {json_number(s['maxInternalIndicator'])}, "
            f"\"earlyElasticSlope_MPa\": {json_number(s['earlyElasticSlope'])}, "
            f"\"analyticalPlaneStrainSlope_MPa\": {json_number(s['analyticalPlaneStrainSlope'])}, "
            f"\"earlyElasticRelativeError\": {json_number(s['earlyElasticRelativeError'])}, "
            f"\"finalReaction_N\": {json_number(s['finalReaction'])}, "
            f"\"finalNominalStress_MPa\": {json_number(s['finalNominalStress'])}, "
            f"\"finalEngineeringStrain\": {json_number(s['finalEngineeringStrain'])}, "
            f"\"finite\": {'true' if s['finite'] else 'false'}}}")
    tail = (
        "\n  ],\n"
        f"  \"acceptance\": {{\"energyToleranceRelative\": {g6(bc.energy_tolerance)}, "
        f"\"netForceTolerance_N\": {g6(bc.net_force_tolerance)}, "
        f"\"minimumPlasticStrain\": {g6(bc.minimum_plastic_strain)}, "
        f"\"kineticToInternalLimit\": {g6(bc.kinetic_to_internal_limit)}}},\n"
        "  \"materialComparisonCaveat\": \"Internal state variables are model-specific observers and are "
        "not mapped to a common bond-breaking rule.\",\n"
        "  \"parameterMatchingPolicy\": \"Only identifiable macroscopic properties are matched; "
        "formulation-specific or hard-coded parameters are not claimed to be equivalent.\",\n"
        "  \"legacyBlockPolicy\": \"Material-independent fixed-width blocks of 256 points; a non-full "
        "final block duplicates its last valid point and discards padded outputs.\"\n}\n")
    return head + ",\n".join(items) + tail


def snapshot_steps(bc: BoundaryCase) -> list:
    """The steps whose fields are written: every ``snapshotEvery`` steps and the last one."""
    marks = set(range(bc.snapshot_every, bc.steps + 1, bc.snapshot_every)) if bc.snapshot_every > 0 else set()
    marks.add(bc.steps)
    return sorted(marks)


def plugin_file(m) -> str:
    """The metadata's plugin_file: the library whose material routine ran."""
    return os.path.basename(m.host_plugin.plugin_path) if m.host_plugin is not None else "libvpd_gpu.so"


SURROGATE_GUESSES = ("network", "hybrid", "warm_start")


def run_boundary_case(path: str, out_dir: str = None, config_root: str = None, precision: int = None,
                      log=print, plugin_dir: str = None, surrogate: str = None) -> int:
    """Runs every material of a boundary-value case file and writes its three output files into
    ``out_dir`` (default: the case's output.directory). Returns 0 when every material passes
    the case's acceptance limits, 2 otherwise (the reference runner's exit status)."""
    from . import Simulation, train_surrogate
    from .case import MATERIAL_SURROGATE
    bc = load_boundary_case(path, config_root, plugin_dir)
    if surrogate is not None:
        if surrogate not in SURROGATE_GUESSES:
            raise ValueError(f"surrogate {surrogate!r}: one of {', '.join(SURROGATE_GUESSES)}")
        for m in bc.materials:
            if m.host_plugin is not None:
                raise ValueError(f"material {m.label}: the surrogate replaces the device Johnson-Cook "
                                 "update, not a host plugin")
    networks = {}  # trained once per set of Johnson-Cook props
    out = out_dir or bc.output_directory
    os.makedirs(out, exist_ok=True)
    summaries = []
    with open(os.path.join(out, "timeseries.csv"), "w") as ts, \
            open(os.path.join(out, "field_snapshots.csv"), "w") as fs:
        ts.write(TIMESERIES_HEADER)
        fs.write(SNAPSHOT_HEADER)
        for m in bc.materials:
            case = m.case if precision is None else m.case.replace(precision=precision)
            if surrogate is not None:
                case = case.replace(material_mode=MATERIAL_SURROGATE)
                if surrogate != "warm_start" and case.props not in networks:
                    networks[case.props] = train_surrogate(case.props)[:2]
            axis = case.load_axis
            started = time.perf_counter()
            chunks, done = [], 0
            with Simulation(case) as sim:
                if m.host_plugin is not None:
                    p = m.host_plugin
                    sim.set_host_vumat(p.plugin_path, p.props, p.nstatev, p.density, cmname=p.cmname,
                                       symbol=p.symbol)
                if m.initial_state:
                    sim.set_initial_state(m.initial_state)
                if m.indicator is not None:
                    sim.set_internal_indicator(*m.indicator)
                if surrogate is not None:
                    w, b = networks.get(case.props, (None, None))
                    sim.set_surrogate(w, b, guess=surrogate, newton_steps=2)
                x0 = sim.field("position")
                lo, hi = observation_bounds(x0, axis, (case.region_layers - 1) * case.spacing,
                                            case.observation_min, case.observation_max)
                for mark in snapshot_steps(bc):
                    chunks.append(sim.step(mark - done))
                    done = mark
                    state = sim.field("state")
                    eqps = state[:, m.eqps_index] if m.eqps_index >= 0 else np.zeros(len(x0))
                    fs.write(snapshot_lines(m.label, mark, chunks[-1][-1, DIAG["time_ms"]], x0,
                                            sim.field("displacement"), sim.field("velocity"),
                                            sim.field("strain")[:, 4 * axis],
                                            sim.field("stress_spatial")[:, 4 * axis], eqps,
                                            sim.field("damage_index")[:, 0],
                                            None if m.indicator is None else indicator_values(m.indicator, state)))
            runtime = time.perf_counter() - started
            rows = np.concatenate(chunks)
            if m.eqps_index < 0:  # no eqps variable: the reference reports 0 (:259-261)
                rows[:, DIAG["max_eqps"]] = 0.0
            for row in rows:
                step = int(row[DIAG["step"]])
                if step % bc.output_every == 0 or step == 1 or step == bc.steps:
                    ts.write(timeseries_line(m.label, row))
            s = summarise(rows, m.elastic_e, m.elastic_nu)
            s.update(runtimeSeconds=runtime, observationMin=lo, observationMax=hi)
            s["pass"] = passes(bc, s)
            summaries.append(s)
            log(f"{bc.name}/{m.label}: particles={case.n_points} runtime_s={g6(runtime)} "
                f"energy_error={g6(s['finalEnergyError'])} max_eqps={g6(s['maxEqps'])} "
                f"pass={'true' if s['pass'] else 'false'}")
    with open(os.path.join(out, "metadata.json"), "w") as f:
        f.write(metadata_text(bc, summaries))
    return 0 if all(s["pass"] for s in summaries) else 2


def main(argv=None) -> int:
    """The reference's vumat_pd_run for its case files (runDemoCaseFromJson,
    DemoCaseRunner.cpp:434-470): dispatches on the case's ``type``."""
    ap = argparse.ArgumentParser(description="Run one of the reference's case files on the GPU.")
    ap.add_argument("case", help="a vumat_pd_boundary_case, vumat_material_point_case or "
                    "vumat_pd_demo_case JSON file")
    ap.add_argument("--out", help="output directory (default: the case's output.directory)")
    ap.add_argument("--config-root", help="directory the material config paths are relative to")
    ap.add_argument("--plugin-dir", help="directory of the materials' VUMAT plugins (default: the "
                    "stock Johnson-Cook plugin is this package's GPU library)")
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64",
                    help="boundary-value cases: FP64 throughout (the drop-in), or FP32 bond sums "
                         "(whose net internal force exceeds the cases' FP64 round-off limit, so "
                         "the verdict reports fail)")
    ap.add_argument("--surrogate", choices=SURROGATE_GUESSES,
                    help="boundary-value cases: the learned Johnson-Cook return map with this guess "
                         "(the network is trained on the GPU first; the VUMAT stays the fallback)")
    args = ap.parse_args(argv)
    try:
        with open(args.case) as f:
            kind = json.load(f).get("type", "vumat_pd_demo")
        if kind == "vumat_material_point_case":
            from .point_runner import run_material_point_case
            return run_material_point_case(args.case, args.out, args.config_root, args.plugin_dir)
        if kind == "vumat_pd_demo_case":
            from .demo_runner import run_demo_case
            return run_demo_case(args.case, args.out, args.config_root, args.plugin_dir)
        if kind != "vumat_pd_boundary_case":
            raise ValueError("Unsupported case type: " + str(kind))
        from .case import PRECISION_FP64, PRECISION_MIXED
        precision = PRECISION_MIXED if args.precision == "mixed" else PRECISION_FP64
        return run_boundary_case(args.case, args.out, args.config_root, precision=precision,
                                 plugin_dir=args.plugin_dir, surrogate=args.surrogate)
    except (ValueError, OSError, RuntimeError) as e:
        print(f"error: {e}", file=sys.stderr)
        return 1


if __name__ == "__main__":
    sys.exit(main())
