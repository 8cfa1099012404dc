"""VUMAT material configs and plugin calls, for the material-point and affine demo case hosts.

``load_vumat_config`` reads a material config (configs/*.json; the reference's
src/config/MaterialConfigJson.cpp:63-101, same defaults and checks) for any VUMAT.
``VumatPlugin.update_block`` makes one call of the plugin's ``vumat_adapter_call`` on up to 256
rows, packing and unpacking its arguments as the reference's adapter does
(VumatMaterialAdapter::updateFixedBlockCached, src/material/VumatMaterialAdapter.cpp:238-362);
``update_point`` is the one-row call of VumatMaterialAdapter::updatePoint (:116-147).

Plugins are found as the reference finds them: ``pluginPath``, or ``plugin`` plus ``.so``,
relative to the plugin directory. Without a plugin directory the stock Johnson-Cook plugin
(``jc_vumat_plugin``) is this package's own library, whose ``vumat_adapter_call`` runs the
Johnson-Cook routine on the GPU; any other plugin then needs a plugin directory.
"""
from __future__ import annotations

import ctypes
import dataclasses
import json
import math
import os

import numpy as np

STOCK_JC_PLUGIN = "jc_vumat_plugin"
IDENTITY = (1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0)


@dataclasses.dataclass
class VumatConfig:
    name: str
    cmname: str
    plugin_path: str
    symbol: str
    nstatev: int
    nfieldv: int
    props: tuple
    density: float
    stress_frame: str


def _library_name(plugin: str) -> str:  # dynamicLibraryName, MaterialConfigJson.cpp:40-50
    if "/" in plugin or "\\" in plugin or "." in plugin:
        return plugin
    return plugin + ".so"


def _number(root, key, default=None):
    if key not in root:
        if default is None:
            raise ValueError(f"material config: {key} is required")
        return default
    value = root[key]
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise ValueError(f"material config: {key} must be a number")
    return value


def load_vumat_config(path: str, plugin_dir: str | None = None) -> VumatConfig:
    """A VUMAT material config, with the plugin resolved (see the module docstring)."""
    with open(path) as f:
        root = json.load(f)
    if root.get("schemaVersion", "1.0") != "1.0":
        raise ValueError("Unsupported VUMAT material schemaVersion: " + str(root.get("schemaVersion")))
    for key in ("name", "cmname"):
        if not isinstance(root.get(key), str):
            raise ValueError(f"material config: {key} is required")
    if root.get("tensorConvention", "legacy_vumat_pd") != "legacy_vumat_pd":
        raise ValueError("Unsupported tensorConvention; explicit mapping is required.")
    frame = root.get("stressFrame", "corotational")
    if frame not in ("corotational", "spatial"):
        raise ValueError("stressFrame must be corotational or spatial.")
    symbol = root.get("symbolName", root.get("symbol", "vumat_adapter_call"))
    ndir, nshr = int(_number(root, "ndir", 3)), int(_number(root, "nshr", 3))
    nstatev, nfieldv = int(_number(root, "nstatev")), int(_number(root, "nfieldv", 1))
    props = root.get("props")
    if not isinstance(props, list) or not all(isinstance(p, (int, float)) and not isinstance(p, bool)
                                              for p in props):
        raise ValueError("material config: props must be a numeric array")
    density = float(_number(root, "density"))
    if ndir != 3 or nshr != 3:
        raise ValueError("The current VUMAT adapter requires ndir=3 and nshr=3.")
    if nstatev < 0 or nfieldv < 0 or density <= 0.0:
        raise ValueError("Invalid VUMAT dimensions or density in: " + path)
    explicit = root.get("pluginPath", "")
    plugin = root.get("plugin", "")
    if not explicit and not plugin:
        raise ValueError("Material config requires either pluginPath or plugin.")
    target = explicit or _library_name(plugin)
    if plugin_dir is None:
        if explicit or plugin != STOCK_JC_PLUGIN:
            if not os.path.isabs(target):
                raise ValueError(f"plugin {target!r}: give the plugin directory to load it")
            resolved = target
        else:
            from . import library_path  # the device Johnson-Cook behind the plugin ABI
            resolved = library_path()
    else:
        resolved = target if os.path.isabs(target) else os.path.join(plugin_dir, target)
    return VumatConfig(name=root["name"], cmname=root["cmname"], plugin_path=resolved,
                       symbol=symbol, nstatev=nstatev, nfieldv=nfieldv,
                       props=tuple(float(p) for p in props), density=density, stress_frame=frame)


def _voigt(t):  # fullTensorToVumatVoigt, TensorVoigtMap.cpp:9-16
    return (t[0], t[4], t[8], 0.5 * (t[5] + t[7]), 0.5 * (t[2] + t[6]), 0.5 * (t[1] + t[3]))


def _full(v):  # vumatVoigtToFullTensor, TensorVoigtMap.cpp:18-20
    return [v[0], v[5], v[4], v[5], v[1], v[3], v[4], v[3], v[2]]


def _defgrad(t):  # fullTensorToVumatDefgrad, TensorVoigtMap.cpp:22-24
    return (t[0], t[4], t[8], t[1], t[5], t[6], t[3], t[7], t[2])


def _voigt_rows(t):
    """fullTensorToVumatVoigt (TensorVoigtMap.cpp:9-16) of each row of t [nb, 9] -> [6, nb]."""
    return np.stack([t[:, 0], t[:, 4], t[:, 8], 0.5 * (t[:, 5] + t[:, 7]), 0.5 * (t[:, 2] + t[:, 6]),
                     0.5 * (t[:, 1] + t[:, 3])])


@dataclasses.dataclass
class PointInput:
    """VumatPointInput (include/VumatTypes.hpp:25-42): full tensors row-major."""
    dt: float
    step_time: float = 0.0
    total_time: float = 0.0
    char_length: float = 1.0
    temperature: float = 0.0
    strain_rate: list = dataclasses.field(default_factory=lambda: [0.0] * 9)
    rel_spin: list = dataclasses.field(default_factory=lambda: [0.0] * 9)
    strain_n: list = dataclasses.field(default_factory=lambda: [0.0] * 9)
    stress_n: list = dataclasses.field(default_factory=lambda: [0.0] * 9)
    stretch_old: list = dataclasses.field(default_factory=lambda: list(IDENTITY))
    stretch_new: list = dataclasses.field(default_factory=lambda: list(IDENTITY))
    defgrad_old: list = dataclasses.field(default_factory=lambda: list(IDENTITY))
    defgrad_new: list = dataclasses.field(default_factory=lambda: list(IDENTITY))
    state_old: list = dataclasses.field(default_factory=list)
    internal_energy_old: float = 0.0
    inelastic_energy_old: float = 0.0

    def copy(self) -> "PointInput":
        return dataclasses.replace(self, **{f.name: list(getattr(self, f.name))
                                            for f in dataclasses.fields(self)
                                            if isinstance(getattr(self, f.name), list)})


@dataclasses.dataclass
class PointResult:
    stress: list          # full tensor, row-major
    state: list
    temperature: float
    internal_energy: float
    inelastic_energy: float


_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)


class VumatPlugin:
    """A loaded plugin and its material config (VumatMaterialAdapter's constructor checks)."""

    def __init__(self, config: VumatConfig):
        if not config.props:
            raise ValueError("VUMAT props cannot be empty.")
        try:
            lib = ctypes.CDLL(config.plugin_path)
        except OSError as e:
            raise RuntimeError(f"Failed to load VUMAT plugin: {e}") from None
        try:
            self._call = getattr(lib, config.symbol)
        except AttributeError:
            raise RuntimeError("Failed to resolve symbol in VUMAT plugin: " + config.symbol) from None
        self._call.restype = None
        self._call.argtypes = [_IP] * 7 + [_DP] * 3 + [ctypes.c_char_p] + [_DP] * 22
        self._lib = lib
        self.config = config
        self._props = np.array(config.props, dtype=np.float64)
        self._cmname = config.cmname.encode()[:80].ljust(80, b" ")

    def update_block(self, *, dt, step_time, total_time, char_length, temperature, strain_rate,
                     rel_spin, stress_n, stretch_old, stretch_new, defgrad_old, defgrad_new,
                     state_old, internal_energy_old, inelastic_energy_old) -> dict:
        """One plugin call on nb <= 256 rows (updateFixedBlockCached, :238-362). Tensors are
        [nb, 9] row-major full tensors, state_old [nb, nstatev], the rest [nb]. Returns the new
        full stress [nb, 9], state [nb, nstatev], temperature and energies [nb]."""
        c = self.config
        if not (math.isfinite(dt) and dt > 0.0):
            raise ValueError("Cached material update requires a positive time step and at most 256 points.")
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        strain_rate, rel_spin, stress_n = f(strain_rate), f(rel_spin), f(stress_n)
        stretch_old, stretch_new = f(stretch_old), f(stretch_new)
        defgrad_old, defgrad_new, state_old = f(defgrad_old), f(defgrad_new), f(state_old)
        nb = strain_rate.shape[0]
        if not 1 <= nb <= 256:
            raise ValueError("Cached material update requires a positive time step and at most 256 points.")
        if state_old.shape != (nb, c.nstatev):
            raise ValueError("stateOld entry size does not match nstatev.")
        # [component][nblock] column-major blocks, as the adapter's work arrays
        strain_inc = np.ascontiguousarray(_voigt_rows(strain_rate) * dt)
        spin = np.ascontiguousarray(np.stack([rel_spin[:, 5], rel_spin[:, 6], rel_spin[:, 1]]))
        stress_old = np.ascontiguousarray(_voigt_rows(stress_n))
        v_old, v_new = np.ascontiguousarray(_voigt_rows(stretch_old)), np.ascontiguousarray(_voigt_rows(stretch_new))
        order = [0, 4, 8, 1, 5, 6, 3, 7, 2]  # fullTensorToVumatDefgrad
        g_old = np.ascontiguousarray(defgrad_old[:, order].T)
        g_new = np.ascontiguousarray(defgrad_new[:, order].T)
        state_cols, field_cols = max(1, c.nstatev), max(1, c.nfieldv)
        st_old = np.zeros((state_cols, nb))
        st_old[:c.nstatev] = state_old.T
        temp_old = f(temperature).copy()
        temp_new = temp_old.copy()
        ei_old, ep_old = f(internal_energy_old).copy(), f(inelastic_energy_old).copy()
        ei_new, ep_new = ei_old.copy(), ep_old.copy()
        stress_new, state_new = np.zeros((6, nb)), np.zeros((state_cols, nb))
        coord, length = np.zeros(3 * nb), f(char_length).copy()
        density = np.full(nb, c.density)
        field_old, field_new = np.zeros(field_cols * nb), np.zeros(field_cols * nb)
        props = self._props.copy()
        ints = [ctypes.c_int(v) for v in (nb, 3, 3, c.nstatev, c.nfieldv, len(c.props), 0)]
        times = [ctypes.c_double(v) for v in (step_time, total_time, dt)]

        def dp(a):
            return a.ctypes.data_as(_DP)

        self._call(*[ctypes.byref(v) for v in ints], *[ctypes.byref(v) for v in times],
                   ctypes.create_string_buffer(self._cmname, 80),
                   dp(coord), dp(length), dp(props), dp(density), dp(strain_inc), dp(spin),
                   dp(temp_old), dp(v_old), dp(g_old), dp(field_old), dp(stress_old),
                   dp(st_old), dp(ei_old), dp(ep_old), dp(temp_new), dp(v_new),
                   dp(g_new), dp(field_new), dp(stress_new), dp(state_new), dp(ei_new), dp(ep_new))
        v = stress_new  # vumatVoigtToFullTensor
        full = np.stack([v[0], v[5], v[4], v[5], v[1], v[3], v[4], v[3], v[2]], axis=1)
        return dict(stress=full, state=state_new[:c.nstatev].T.copy(), temperature=temp_new,
                    internal_energy=ei_new, inelastic_energy=ep_new)

    def update_point(self, p: PointInput) -> PointResult:
        """One point through the plugin: updatePoint as a one-row block (:116-147), packed
        directly (a host loop calls it once per evaluation)."""
        c = self.config
        if not (math.isfinite(p.dt) and p.dt > 0.0):
            raise ValueError("VUMAT update requires dt > 0.")
        if len(p.state_old) != c.nstatev:
            raise ValueError("stateOld entry size does not match nstatev.")

        def arr(values):
            return np.array(values, dtype=np.float64)

        field_cols, state_cols = max(1, c.nfieldv), max(1, c.nstatev)
        stress_old = arr(_voigt(p.stress_n))
        strain_inc = arr([v * p.dt for v in _voigt(p.strain_rate)])
        spin = arr((p.rel_spin[5], p.rel_spin[6], p.rel_spin[1]))
        stretch_old, stretch_new = arr(_voigt(p.stretch_old)), arr(_voigt(p.stretch_new))
        defgrad_old, defgrad_new = arr(_defgrad(p.defgrad_old)), arr(_defgrad(p.defgrad_new))
        state_old = np.zeros(state_cols)
        state_old[:c.nstatev] = p.state_old
        temp_old, temp_new = arr([p.temperature]), arr([p.temperature])
        ei_old, ep_old = arr([p.internal_energy_old]), arr([p.inelastic_energy_old])
        ei_new, ep_new = arr([p.internal_energy_old]), arr([p.inelastic_energy_old])
        stress_new, state_new = np.zeros(6), np.zeros(state_cols)
        coord, char_length, density = np.zeros(3), arr([p.char_length]), arr([c.density])
        field_old, field_new = np.zeros(field_cols), np.zeros(field_cols)
        props = self._props.copy()
        ints = [ctypes.c_int(v) for v in (1, 3, 3, c.nstatev, c.nfieldv, len(c.props), 0)]
        times = [ctypes.c_double(v) for v in (p.step_time, p.total_time, p.dt)]

        def dp(a):
            return a.ctypes.data_as(_DP)

        self._call(*[ctypes.byref(v) for v in ints], *[ctypes.byref(v) for v in times],
                   ctypes.create_string_buffer(self._cmname, 80),
                   dp(coord), dp(char_length), dp(props), dp(density), dp(strain_inc), dp(spin),
                   dp(temp_old), dp(stretch_old), dp(defgrad_old), dp(field_old), dp(stress_old),
                   dp(state_old), dp(ei_old), dp(ep_old), dp(temp_new), dp(stretch_new),
                   dp(defgrad_new), dp(field_new), dp(stress_new), dp(state_new), dp(ei_new),
                   dp(ep_new))
        return PointResult(stress=_full(stress_new.tolist()), state=state_new[:c.nstatev].tolist(),
                           temperature=float(temp_new[0]), internal_energy=float(ei_new[0]),
                           inelastic_energy=float(ep_new[0]))
