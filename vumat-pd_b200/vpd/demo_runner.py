"""The reference's affine correspondence-PD demo case (``"type": "vumat_pd_demo_case"``; its
examples/affine_bar_elastic.json and affine_shear_elastic.json). A small PD patch is put under
an affine displacement field, with one quasi-static update per step. Each step is checked
against the exact deformation gradient and the elastic reference stress, and the run is written
as the reference's ``timeseries.csv``, ``field_final.csv`` and ``metadata.json``
(DemoCaseRunner.cpp:295-491).

The PD work runs on the GPU through this package's module functions:
  * the neighbour list and K^-1,
  * the deformation gradients and the corotational kinematics,
  * critical-stretch bond damage,
  * the force density.
The material is the VUMAT-PD bridge (VumatPdCorrespondenceMaterial::update,
VumatPdCorrespondenceMaterial.cpp:72-176). It runs the material's plugin on 256-row blocks
(``vpd.vumat_plugin``). The stock Johnson-Cook plugin is this package's library, so that routine
also runs on the GPU.

The CSV files use the stream's default 6 significant digits and the metadata 16, as the
reference writes them.
"""
from __future__ import annotations

import math
import os

import numpy as np

from . import (build_neighbor_list, corotational_update, damage_update, deformation_gradients,
               force_density, shape_tensor_inverse)
from .point_runner import AffineCase, load_affine_case, state_indicator
from .vumat_plugin import IDENTITY, VumatPlugin

_DEVICE = "cuda"
BLOCK = 256  # rows of one plugin call (VumatPdCorrespondenceMaterial.cpp:90)

TIMESERIES_HEADER = ("material,step,time,applied_strain,max_f_error,avg_raw_stress_xx,"
                     "avg_effective_stress_xx,avg_raw_stress_xy,avg_effective_stress_xy,"
                     "elastic_reference_stress_xx,elastic_reference_stress_xy,"
                     "max_stress_reference_error,max_damage,avg_damage,net_force_x,"
                     "net_force_y,net_force_z,net_force_norm,left_reaction_x,"
                     "right_reaction_x,avg_internal_indicator,max_internal_indicator,finite\n")
FIELD_HEADER = ("material,particle,x0,y0,z0,ux,uy,uz,x,y,z,"
                "Fxx,Fxy,Fxz,Fyx,Fyy,Fyz,Fzx,Fzy,Fzz,"
                "strain_xx,raw_stress_xx,effective_stress_xx,damage,"
                "internal_indicator,force_x,force_y,force_z\n")


def g6(x: float) -> str:
    return "%g" % x


def g16(x: float) -> str:
    return "%.16g" % x


def _max(a: float, b: float) -> float:  # std::max: a unless a < b
    return b if a < b else a


def make_patch(nx: int, ny: int, nz: int, h: float):
    """makeParticlePatch (Geometry.cpp:10-34): lattice positions [n,3] and the trapezoidal
    volumes [n] (halved on each face)."""
    yoff = 0.5 * float(ny - 1) * h
    zoff = 0.5 * float(nz - 1) * h
    volume = h * h * h
    pos, vol = [], []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                pos.append((float(i) * h, float(j) * h - yoff, float(k) * h - zoff))
                vol.append(volume * (0.5 if i in (0, nx - 1) else 1.0) * (0.5 if j in (0, ny - 1) else 1.0)
                           * (0.5 if k in (0, nz - 1) else 1.0))
    return np.array(pos), np.array(vol)


def _multiply(a, b):
    """Row-major 3x3 products of each row of a, b [n,9], summed in the reference's order
    (CorotationalKinematics.cpp:27-34)."""
    out = np.zeros_like(a)
    for i in range(3):
        for j in range(3):
            acc = np.zeros(a.shape[0])
            for k in range(3):
                acc = acc + a[:, 3 * i + k] * b[:, 3 * k + j]
            out[:, 3 * i + j] = acc
    return out


def rotate_to_spatial(stress, rotation):
    """rotateCorotationalStressToSpatial: R (sigma R^T) per row (CorotationalKinematics.cpp:137-139)."""
    rt = rotation[:, [0, 3, 6, 1, 4, 7, 2, 5, 8]]
    return _multiply(rotation, _multiply(stress, rt))


def _max_principal(t) -> float:
    """maxPrincipalStrainSymmetric3x3 (TensorVoigtMap.cpp:35-71) of one row-major tensor."""
    a, b, c = t[0], 0.5 * (t[1] + t[3]), 0.5 * (t[2] + t[6])
    d, e, f = t[4], 0.5 * (t[5] + t[7]), t[8]
    p1 = b * b + c * c + e * e
    if p1 == 0.0:
        return max(a, d, f)
    q = (a + d + f) / 3.0
    a11, a22, a33 = a - q, d - q, f - q
    p = math.sqrt((a11 * a11 + a22 * a22 + a33 * a33 + 2.0 * p1) / 6.0)
    inv = 1.0 / p
    b11, b12, b13, b22, b23, b33 = a11 * inv, b * inv, c * inv, a22 * inv, e * inv, a33 * inv
    det = b11 * (b22 * b33 - b23 * b23) - b12 * (b12 * b33 - b23 * b13) + b13 * (b12 * b23 - b22 * b13)
    r = min(max(det / 2.0, -1.0), 1.0)
    phi = math.acos(r) / 3.0
    e1 = q + 2.0 * p * math.cos(phi)
    e3 = q + 2.0 * p * math.cos(phi + 2.0 * math.pi / 3.0)
    e2 = 3.0 * q - e1 - e3
    return max(e1, e2, e3)


class HostBridge:
    """VumatPdCorrespondenceMaterial with its history in host arrays: the kinematics on the
    GPU (vpd.corotational_update), the plugin on 256-row blocks, the short last block padded
    with its last row (:93-177). ``initialize`` is :47-70."""

    def __init__(self, plugin: VumatPlugin, char_length: float, temperature: float, initial_state,
                 defgrad0):
        import torch
        n = defgrad0.shape[0]
        self.plugin, self.char_length = plugin, char_length
        self.Fn = defgrad0.clone()
        eye = torch.tensor(IDENTITY, dtype=torch.float64, device=defgrad0.device)
        self.Vn = eye.repeat(n, 1).contiguous()
        self.Rn = eye.repeat(n, 1).contiguous()
        self.sig = np.zeros((n, 9))               # corotational stress (rawStressN)
        self.state = np.tile(np.asarray(initial_state, dtype=np.float64), (n, 1)).reshape(n, -1)
        self.temp = np.full(n, temperature)
        self.eI, self.eP = np.zeros(n), np.zeros(n)

    def update(self, F, dt: float, step_time: float):
        """One increment; returns (spatial stress [n,9], strain [n,9]) on the host."""
        kin = corotational_update(self.Fn, F, self.Vn, self.Rn, dt)
        h = {k: v.cpu().numpy() for k, v in kin.items()}
        Fn, Fh, Vn = self.Fn.cpu().numpy(), F.cpu().numpy(), self.Vn.cpu().numpy()
        n = Fh.shape[0]
        sig, state = np.empty_like(self.sig), np.empty_like(self.state)
        temp, eI, eP = np.empty(n), np.empty(n), np.empty(n)
        for begin in range(0, n, BLOCK):
            end = min(begin + BLOCK, n)
            rows = np.concatenate([np.arange(begin, end), np.full(BLOCK - (end - begin), end - 1)])
            r = self.plugin.update_block(
                dt=dt, step_time=step_time, total_time=step_time,
                char_length=np.full(BLOCK, self.char_length), temperature=self.temp[rows],
                strain_rate=h["rate_of_deformation"][rows], rel_spin=h["relative_spin"][rows],
                stress_n=self.sig[rows], stretch_old=Vn[rows], stretch_new=h["left_stretch"][rows],
                defgrad_old=Fn[rows], defgrad_new=Fh[rows], state_old=self.state[rows],
                internal_energy_old=self.eI[rows], inelastic_energy_old=self.eP[rows])
            count = end - begin
            sig[begin:end] = r["stress"][:count]
            state[begin:end] = r["state"][:count]
            temp[begin:end] = r["temperature"][:count]
            eI[begin:end] = r["internal_energy"][:count]
            eP[begin:end] = r["inelastic_energy"][:count]
        spatial = rotate_to_spatial(sig, h["rotation"])
        self.Fn, self.Vn, self.Rn = F.clone(), kin["left_stretch"], kin["rotation"]
        self.sig, self.state, self.temp, self.eI, self.eP = sig, state, temp, eI, eP
        return spatial, h["strain"]


def _elastic_references(e: float, nu: float, load: float, shear: bool):
    """referenceStressXx / referenceStressXy (DemoCaseRunner.cpp:49-60, 145-157)."""
    mu = e / (2.0 * (1.0 + nu))
    if shear:
        return 0.0, mu * load
    lam = e * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return (lam + 2.0 * mu) * load, 0.0


def run_material(case: AffineCase, m, time_lines: list, field_lines: list) -> dict:
    """runMaterial (DemoCaseRunner.cpp:295-431) for one material."""
    import torch
    if case.max_strain == 0.0:
        raise ValueError("Affine displacement boundary condition requires maxStrain.")
    shear = case.mode == "simple_shear_xy"
    pos, vol = make_patch(case.nx, case.ny, case.nz, case.spacing)
    n = pos.shape[0]
    X = torch.tensor(pos, dtype=torch.float64, device=_DEVICE)
    V = torch.tensor(vol, dtype=torch.float64, device=_DEVICE)
    row_ptr, col = build_neighbor_list(X, case.horizon)
    kinv = shape_tensor_inverse(X, V, row_ptr, col)
    zero = torch.zeros((n, 3), dtype=torch.float64, device=_DEVICE)
    bridge = HostBridge(VumatPlugin(m.config), case.spacing, m.reference_temperature,
                        m.initial_state or [0.0] * m.config.nstatev,
                        deformation_gradients(X, zero, V, row_ptr, col, kinv))
    bonds = torch.zeros(max(int(col.shape[0]), 1), dtype=torch.float64, device=_DEVICE)
    point_damage = np.zeros(n)
    if case.damage_model == "critical_stretch" and not case.damage_initiation > 0.0:
        raise ValueError("critical_stretch requires initiation > 0.")
    if case.damage_model in ("eqps_threshold", "max_principal_strain") and \
            not case.damage_failure - case.damage_initiation > 0.0:
        raise ValueError("SimpleDamageModel requires failure > initiation.")
    if case.damage_model not in ("none", "critical_stretch", "eqps_threshold", "max_principal_strain"):
        raise ValueError("Unsupported simple damage mode: " + case.damage_model)
    if case.damage_model == "eqps_threshold" and m.config.nstatev < 2:
        raise ValueError("eqpsStateIndex is outside the VUMAT state vector.")
    min_x, max_x = np.finfo(float).max, -np.finfo(float).max
    for x in pos[:, 0]:
        min_x = x if x < min_x else min_x
        max_x = max_x if x < max_x else x
    s = dict(key=m.label, reference=m.reference, maxFError=0.0, maxStressReferenceError=0.0,
             maxNetForceNorm=0.0, maxDamage=0.0, finite=True)
    dt, steps = case.dt, case.steps
    for step in range(1, steps + 1):
        load = case.max_strain * float(step) / float(steps)
        disp = np.zeros((n, 3))
        disp[:, 0] = load * pos[:, 1] if shear else load * pos[:, 0]
        U = torch.tensor(disp, dtype=torch.float64, device=_DEVICE)
        exact = [1.0, load if shear else 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0]
        if not shear:
            exact[0] = 1.0 + load
        ref_xx, ref_xy = _elastic_references(m.elastic_e, m.elastic_nu, load, shear)
        F = deformation_gradients(X, U, V, row_ptr, col, kinv)
        raw, strain = bridge.update(F, dt, float(step - 1) * dt)
        effective, damage = raw, np.zeros(n)
        if case.damage_model == "critical_stretch":  # PdSimpleDamage.cpp:59-82
            damage = damage_update(X, U, V, row_ptr, col, case.damage_initiation, case.damage_failure,
                                   bonds).cpu().numpy()
        elif case.damage_model != "none":  # SimpleDamageModel.cpp:14-50
            factor = np.empty(n)
            for i in range(n):
                metric = (bridge.state[i, 1] if case.damage_model == "eqps_threshold"
                          else _max_principal(strain[i]))
                t = (metric - case.damage_initiation) / (case.damage_failure - case.damage_initiation)
                d = _max(point_damage[i], 0.0 if t < 0.0 else (1.0 if 1.0 < t else t))
                point_damage[i] = d
                factor[i] = 0.0 if (case.damage_deletion and d >= 1.0) else 1.0 - min(max(d, 0.0), 1.0)
            effective, damage = raw * factor[:, None], point_damage.copy()
        force = force_density(X, V, row_ptr, col, kinv, F,
                              torch.tensor(effective, dtype=torch.float64, device=_DEVICE).contiguous(),
                              bonds).cpu().numpy()
        Fh = F.cpu().numpy()
        max_f_error = 0.0
        for v in np.abs(Fh - np.array(exact)[None, :]).ravel():
            max_f_error = _max(max_f_error, v)
        raw_sum = raw_xy_sum = eff_sum = eff_xy_sum = damage_sum = 0.0
        max_damage = max_ref_error = 0.0
        finite = s["finite"]
        for i in range(n):
            finite = (finite and np.isfinite(raw[i]).all() and np.isfinite(effective[i]).all()
                      and np.isfinite(force[i]).all() and math.isfinite(damage[i]))
            raw_sum += raw[i, 0]
            eff_sum += effective[i, 0]
            xy = 0.5 * (raw[i, 1] + raw[i, 3])
            eff_xy = 0.5 * (effective[i, 1] + effective[i, 3])
            raw_xy_sum += xy
            eff_xy_sum += eff_xy
            damage_sum += damage[i]
            max_damage = _max(max_damage, damage[i])
            max_ref_error = _max(max_ref_error, _max(abs(raw[i, 0] - ref_xx), abs(xy - ref_xy)))
        count = float(n)
        net = [0.0, 0.0, 0.0]
        left = right = 0.0
        for i in range(n):  # summarizeForces, :206-225
            for d in range(3):
                net[d] += force[i, d] * vol[i]
            if abs(pos[i, 0] - min_x) < 1.0e-12:
                left += force[i, 0] * vol[i]
            if abs(pos[i, 0] - max_x) < 1.0e-12:
                right += force[i, 0] * vol[i]
        net_norm = math.sqrt(net[0] * net[0] + net[1] * net[1] + net[2] * net[2])
        indicators = [state_indicator(m, bridge.state[i]) for i in range(n)]
        ind_sum, ind_max = 0.0, 0.0
        for v in indicators:
            ind_sum += v
            ind_max = _max(ind_max, v)
        ind_avg = ind_sum / count
        s["maxFError"] = _max(s["maxFError"], max_f_error)
        s["maxStressReferenceError"] = _max(s["maxStressReferenceError"], max_ref_error)
        s["maxNetForceNorm"] = _max(s["maxNetForceNorm"], net_norm)
        s["maxDamage"] = _max(s["maxDamage"], max_damage)
        s["finite"] = (finite and all(math.isfinite(v) for v in net) and np.isfinite(bridge.state).all()
                       and math.isfinite(ind_avg) and math.isfinite(ind_max) and math.isfinite(left)
                       and math.isfinite(right))
        time_lines.append(",".join([m.label, str(step)] + [g6(v) for v in (
            step * dt, load, max_f_error, raw_sum / count, eff_sum / count, raw_xy_sum / count,
            eff_xy_sum / count, ref_xx, ref_xy, max_ref_error, max_damage, damage_sum / count,
            net[0], net[1], net[2], net_norm, left, right, ind_avg, ind_max)]
            + ["1" if s["finite"] else "0"]) + "\n")
    for i in range(n):  # the final fields, :405-419
        head = [m.label, str(i)] + [g6(v) for v in (*pos[i], *disp[i], *(pos[i] + disp[i]))]
        tail = [g6(v) for v in (strain[i, 0], raw[i, 0], effective[i, 0], damage[i], indicators[i],
                                *force[i])]
        field_lines.append(",".join(head) + "," + "".join(g6(v) + "," for v in Fh[i]) + ",".join(tail) + "\n")
    return s


def _escape(text: str) -> str:  # jsonEscape, :101-124
    return (text.replace("\\", "\\\\").replace('"', '\\"').replace("\n", "\\n")
            .replace("\r", "\\r").replace("\t", "\\t"))


def metadata_text(case: AffineCase, summaries: list) -> str:
    """writeMetadata (DemoCaseRunner.cpp:227-293)."""
    max_f = max_ref = max_net = max_dmg = 0.0
    finite = True
    for s in summaries:
        max_f = _max(max_f, s["maxFError"])
        if s["reference"]:
            max_ref = _max(max_ref, s["maxStressReferenceError"])
        max_net = _max(max_net, s["maxNetForceNorm"])
        max_dmg = _max(max_dmg, s["maxDamage"])
        finite = finite and s["finite"]
    passed = (finite and max_f < case.deformation_gradient_tolerance
              and (not summaries or max_ref < case.reference_stress_tolerance)
              and max_net < case.net_force_tolerance)
    b = lambda v: "true" if v else "false"  # noqa: E731
    notes = case.scope + (". Checks: " + "; ".join(case.checks) if case.checks else "")
    text = ("{\n"
            f"  \"name\": \"{case.name}\",\n  \"status\": \"{'pass' if passed else 'fail'}\",\n"
            f"  \"scope\": \"{case.scope}\",\n  \"particles\": {case.nx * case.ny * case.nz},\n"
            f"  \"steps\": {case.steps},\n  \"maxDeformationGradientError\": {g16(max_f)},\n"
            f"  \"maxReferenceStressError\": {g16(max_ref)},\n  \"maxJcRawStressError\": {g16(max_ref)},\n"
            f"  \"maxNetForceNorm\": {g16(max_net)},\n  \"maxDamage\": {g16(max_dmg)},\n"
            f"  \"allValuesFinite\": {b(finite)},\n"
            f"  \"tolerances\": {{\"deformationGradientAbsolute\": {g16(case.deformation_gradient_tolerance)}, "
            f"\"referenceStressAbsolute\": {g16(case.reference_stress_tolerance)}, "
            f"\"netForceAbsolute\": {g16(case.net_force_tolerance)}}},\n"
            f"  \"notes\": \"{_escape(notes)}\",\n  \"checks\": [\n")
    text += "".join(f"    \"{c}\"" + ("\n" if k + 1 == len(case.checks) else ",\n") for k, c in enumerate(case.checks))
    text += "  ],\n  \"materials\": [\n"
    text += "".join(
        f"    {{\"name\": \"{s['key']}\", \"reference\": {b(s['reference'])}, "
        f"\"maxDeformationGradientError\": {g16(s['maxFError'])}, "
        f"\"maxStressReferenceError\": {g16(s['maxStressReferenceError'])}, "
        f"\"maxNetForceNorm\": {g16(s['maxNetForceNorm'])}, \"maxDamage\": {g16(s['maxDamage'])}, "
        f"\"finite\": {b(s['finite'])}}}" + ("\n" if k + 1 == len(summaries) else ",\n")
        for k, s in enumerate(summaries))
    return text + "  ]\n}\n"


def run_demo_case(path: str, out_dir: str | None = None, config_root: str | None = None,
                  plugin_dir: str | None = None, log=print) -> int:
    """Runs the case and writes its files; 0 when every material passes, 2 otherwise (:434-491)."""
    case = load_affine_case(path, "vumat_pd_demo_case", config_root, plugin_dir)
    out = out_dir or case.output_directory
    os.makedirs(out, exist_ok=True)
    time_lines, field_lines = [TIMESERIES_HEADER], [FIELD_HEADER]
    summaries = [run_material(case, m, time_lines, field_lines) for m in case.materials]
    with open(os.path.join(out, "timeseries.csv"), "w") as f:
        f.write("".join(time_lines))
    with open(os.path.join(out, "field_final.csv"), "w") as f:
        f.write("".join(field_lines))
    with open(os.path.join(out, "metadata.json"), "w") as f:
        f.write(metadata_text(case, summaries))
    passed = True
    for s in summaries:
        passed = (passed and s["finite"] and s["maxFError"] < case.deformation_gradient_tolerance
                  and s["maxNetForceNorm"] < case.net_force_tolerance)
        if s["reference"]:
            passed = passed and s["maxStressReferenceError"] < case.reference_stress_tolerance
        log(f"{s['key']}: max_f_error={s['maxFError']:g} max_stress_reference_error="
            f"{s['maxStressReferenceError']:g} max_damage={s['maxDamage']:g} max_net_force_norm="
            f"{s['maxNetForceNorm']:g} finite={'true' if s['finite'] else 'false'}")
    log(f"VUMAT-PD demo case written to {out}")
    return 0 if passed else 2
