"""Case definitions: the ``vpd_case`` C struct and the tensile-bar workloads.

``VpdCase`` mirrors ``struct vpd_case`` in include/vpd_gpu.h field for field; it carries
the parts of the reference's DemoCaseConfig (include/DemoConfig.hpp:71-167) that the PD
increment reads, in the reference's mm-ms-N-MPa units.

Workloads:
  * ``pd_coarse()`` -- the reference's archived regional JC case,
    benchmarks/tensile3d/cases/pd_coarse.json with configs/johnson_cook.json;
  * ``tensile_bar(1|2|3)`` -- steel Johnson-Cook tensile bars pulled by velocity-ramp grips:
    40x10x10 (h=0.5 mm), 200x50x50 and 400x50x50 (h=0.1 mm, the last jittered by
    +-0.05 h, horizon 4.015 h, adiabatic heating), dt = 0.8 h / c_p.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math

BC_SMOOTH_DISPLACEMENT = 0
BC_VELOCITY_RAMP = 1
DAMAGE_NONE = 0
DAMAGE_CRITICAL_STRETCH = 1
DAMAGE_EQPS_THRESHOLD = 2
DAMAGE_MAX_PRINCIPAL_STRAIN = 3
PRECISION_FP64 = 0
PRECISION_MIXED = 1
MATERIAL_VUMAT = 0
MATERIAL_SURROGATE = 1

DIAG_COLUMNS = (
    "step", "time_ms", "load_displacement_mm", "load_velocity_mm_per_ms", "reaction_force_N",
    "engineering_strain", "lateral_strain", "nominal_stress_MPa", "average_axial_strain",
    "average_axial_stress_MPa", "max_eqps", "max_internal_indicator", "kinetic_energy_Nmm",
    "internal_energy_Nmm", "external_work_Nmm", "relative_energy_error",
    "net_internal_force_N", "finite", "plastic_points", "fallback_points")
DIAG = {name: i for i, name in enumerate(DIAG_COLUMNS)}

FIELDS = ("position", "volume", "displacement", "velocity", "acceleration", "defgrad",
          "stress_corotational", "stress_spatial", "strain", "rotation", "left_stretch",
          "state", "temperature", "energy_internal", "energy_inelastic", "damage_index",
          "force_density", "shape_inverse")
FIELD = {name: i for i, name in enumerate(FIELDS)}
FIELD_WIDTH = {"position": 3, "volume": 1, "displacement": 3, "velocity": 3,
               "acceleration": 3, "defgrad": 9, "stress_corotational": 9,
               "stress_spatial": 9, "strain": 9, "rotation": 9, "left_stretch": 9,
               "temperature": 1, "energy_internal": 1, "energy_inelastic": 1,
               "damage_index": 1, "force_density": 3, "shape_inverse": 9}


class VpdCase(ctypes.Structure):
    """``struct vpd_case`` (include/vpd_gpu.h)."""
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("spacing", ctypes.c_double), ("horizon", ctypes.c_double),
        ("jitter", ctypes.c_double), ("jitter_seed", ctypes.c_uint64),
        ("dt", ctypes.c_double), ("density", ctypes.c_double),
        ("bc_mode", ctypes.c_int32), ("load_axis", ctypes.c_int32),
        ("region_layers", ctypes.c_int32), ("plane_strain", ctypes.c_int32),
        ("amplitude", ctypes.c_double), ("rise_time", ctypes.c_double),
        ("grip_velocity", ctypes.c_double), ("ramp_time", ctypes.c_double),
        ("observation_min", ctypes.c_double), ("observation_max", ctypes.c_double),
        ("props", ctypes.c_double * 14), ("nstatev", ctypes.c_int32),
        ("reference_temperature", ctypes.c_double),
        ("damage_mode", ctypes.c_int32), ("damage_initiation", ctypes.c_double),
        ("damage_failure", ctypes.c_double),
        ("precision", ctypes.c_int32), ("material_mode", ctypes.c_int32),
        ("damage_deletion", ctypes.c_int32),
    ]


@dataclasses.dataclass
class Case:
    """A regional boundary-value case; ``to_c()`` gives the ``vpd_case`` struct."""
    name: str
    nx: int
    ny: int
    nz: int
    spacing: float
    horizon: float
    dt: float
    steps: int
    density: float
    props: tuple
    jitter: float = 0.0
    jitter_seed: int = 0
    bc_mode: int = BC_VELOCITY_RAMP
    load_axis: int = 0
    region_layers: int = 3
    plane_strain: bool = False
    amplitude: float = 0.0
    rise_time: float = 0.0
    grip_velocity: float = 0.0
    ramp_time: float = 0.0
    observation_min: float = math.nan
    observation_max: float = math.nan
    nstatev: int = 6
    reference_temperature: float = 293.0
    damage_mode: int = DAMAGE_NONE
    damage_initiation: float = 0.0
    damage_failure: float = 0.0
    precision: int = PRECISION_FP64
    material_mode: int = MATERIAL_VUMAT
    damage_deletion: bool = False

    @property
    def n_points(self) -> int:
        return self.nx * self.ny * self.nz

    def replace(self, **kw) -> "Case":
        return dataclasses.replace(self, **kw)

    def to_c(self) -> VpdCase:
        c = VpdCase()
        for f in dataclasses.fields(self):
            if f.name in ("name", "steps", "props"):
                continue
            value = getattr(self, f.name)
            setattr(c, f.name, int(value) if isinstance(value, bool) else value)
        if len(self.props) != 14:
            raise ValueError("Johnson-Cook needs 14 props")
        for i, p in enumerate(self.props):
            c.props[i] = float(p)
        return c


# configs/johnson_cook.json (props order: materials/examples/JohnsonCook.f90:9)
REFERENCE_JC_PROPS = (210000.0, 0.30, 350.0, 500.0, 0.025, 0.36, 1.0, 1.0, 293.0, 1793.0,
                      7800.0, 0.9, 500.0, 1.0)


def pd_coarse(steps: int = 4800) -> Case:
    """benchmarks/tensile3d/cases/pd_coarse.json: 51x11x3 nodes, h=2 mm, delta=6 mm,
    half-cosine displacement of the right band to 2 mm over 0.12 ms."""
    return Case(name="pd_coarse", nx=51, ny=11, nz=3, spacing=2.0, horizon=6.0,
                dt=2.4999999999999998e-05, steps=steps, density=0.0078,
                props=REFERENCE_JC_PROPS, bc_mode=BC_SMOOTH_DISPLACEMENT, region_layers=2,
                amplitude=2.0, rise_time=0.12, observation_min=2.0, observation_max=98.0)


# Steel Johnson-Cook in solver units: E, nu, A, B, C, n, m, rate0 (1/s = 1e-3 /ms), Tref,
# Tmelt, rho (kg/m^3, energy bookkeeping only), beta, Cp, workToHeat.
def steel_props(work_to_heat: float = 1.0) -> tuple:
    return (200000.0, 0.3, 350.0, 275.0, 0.022, 0.36, 1.0, 1.0e-3, 293.0, 1793.0, 7850.0,
            0.9, 477.0, work_to_heat)


STEEL_DENSITY = 7850.0e-6  # kg/m^3 * 1e-6 -> N ms^2 / mm^4


def stable_dt(spacing: float, props: tuple = None, density: float = STEEL_DENSITY,
              fraction: float = 0.8) -> float:
    """fraction * h / c_p with the P-wave speed c_p = sqrt(E(1-nu) / (rho(1+nu)(1-2nu)))."""
    props = props or steel_props()
    e, nu = props[0], props[1]
    cp = math.sqrt(e * (1.0 - nu) / (density * (1.0 + nu) * (1.0 - 2.0 * nu)))
    return fraction * spacing / cp


def tensile_bar(config: int, **overrides) -> Case:
    """The steel tensile bars. Grips are three lattice planes at each x end moving apart at
    grip_velocity (mm/ms, 1 mm/ms = 1 m/s), ramped linearly over the first 200 steps."""
    if config == 1:
        nx, ny, nz, h, ratio, steps, v = 40, 10, 10, 0.5, 3.015, 2000, 1.0
        extra = dict(damage_mode=DAMAGE_NONE)
        props = steel_props()
    elif config == 2:
        nx, ny, nz, h, ratio, steps, v = 200, 50, 50, 0.1, 3.015, 5000, 1.0
        extra = dict(damage_mode=DAMAGE_CRITICAL_STRETCH, damage_initiation=0.02,
                     precision=PRECISION_MIXED)
        props = steel_props()
    elif config == 3:
        nx, ny, nz, h, ratio, steps, v = 400, 50, 50, 0.1, 4.015, 10000, 5.0
        extra = dict(damage_mode=DAMAGE_CRITICAL_STRETCH, damage_initiation=0.02,
                     jitter=0.05, jitter_seed=20261203, precision=PRECISION_MIXED)
        props = steel_props(work_to_heat=1.0e6)
    else:
        raise ValueError(f"unknown tensile bar config {config}")
    dt = stable_dt(h, props)
    case = Case(name=f"tensile_bar_{config}", nx=nx, ny=ny, nz=nz, spacing=h,
                horizon=ratio * h, dt=dt, steps=steps, density=STEEL_DENSITY, props=props,
                bc_mode=BC_VELOCITY_RAMP, region_layers=3, grip_velocity=v,
                ramp_time=200 * dt, **extra)
    return case.replace(**overrides) if overrides else case
