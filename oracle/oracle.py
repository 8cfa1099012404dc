"""ORACLE / TEST INFRASTRUCTURE ONLY -- ctypes access to the CPU checkers.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU baseline, as the checker,
never as the thing measured or shipped.

  * ``OracleSim`` and the module functions wrap oracle/_ref/libvpd_oracle.so, the C
    restatement of the reference's PD increment (vpd_oracle.c, jc_vumat.c, case_ext.c).
  * ``RefSim`` wraps oracle/_ref/libvpd_refharness.so, which runs the reference library
    itself (its C++ sources compiled by oracle/Makefile) with the restated JC plugin.

Both are built by ``make -C oracle``; on a machine without the reference sources only the
prebuilt oracle/_ref files are used.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "vumat-pd_b200"))
from vpd.case import FIELD, FIELD_WIDTH, VpdCase  # noqa: E402

_D = ctypes.POINTER(ctypes.c_double)
_I64 = ctypes.POINTER(ctypes.c_int64)
_I32 = ctypes.POINTER(ctypes.c_int32)
DIAG_COLS = 20


def _lib(name):
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
    return ctypes.CDLL(path)


def _dp(a):
    return a.ctypes.data_as(_D)


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        lib = _lib("libvpd_oracle.so")
        lib.vo_create.restype = ctypes.c_void_p
        lib.vo_create.argtypes = [ctypes.POINTER(VpdCase), _D, _D, ctypes.POINTER(ctypes.c_int)]
        lib.vo_step.argtypes = [ctypes.c_void_p, ctypes.c_int32, _D]
        lib.vo_get.argtypes = [ctypes.c_void_p, ctypes.c_int32, _D]
        lib.vo_destroy.argtypes = [ctypes.c_void_p]
        lib.vo_num_points.restype = ctypes.c_int64
        lib.vo_num_points.argtypes = [ctypes.c_void_p]
        lib.vo_num_bonds.restype = ctypes.c_int64
        lib.vo_num_bonds.argtypes = [ctypes.c_void_p]
        lib.vo_neighbors.argtypes = [ctypes.c_void_p, _I64, _I32]
        lib.vo_neighbor_count.restype = ctypes.c_int64
        lib.vo_neighbor_count.argtypes = [_D, ctypes.c_int64, ctypes.c_double, _I64]
        lib.vo_neighbor_fill.argtypes = [_D, ctypes.c_int64, ctypes.c_double, _I64, _I32]
        lib.vo_shape_inverse.argtypes = [ctypes.c_int64, _D, _D, _I64, _I32, _D]
        lib.vo_deformation.argtypes = [ctypes.c_int64, _D, _D, _D, _I64, _I32, _D, _D]
        lib.vo_force.argtypes = [ctypes.c_int64, _D, _D, _I64, _I32, _D, _D, _D, _D, _D]
        lib.vo_corotational.argtypes = [ctypes.c_int64, _D, _D, _D, _D, ctypes.c_double,
                                        _D, _D, _D, _D, _D]
        lib.vo_material_update.argtypes = [ctypes.c_int64, _D, ctypes.c_int32, ctypes.c_double,
                                           _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D]
        lib.vo_damage.argtypes = [ctypes.c_int64, _D, _D, _D, _I64, _I32, ctypes.c_double,
                                  ctypes.c_double, _D, _D]
        lib.vo_jitter_value.restype = ctypes.c_double
        lib.vo_jitter_value.argtypes = [ctypes.c_uint64, ctypes.c_int64, ctypes.c_int,
                                        ctypes.c_double]
        lib.vo_ramp.argtypes = [ctypes.POINTER(VpdCase), ctypes.c_double, _D]
        lib.vo_set_perturbation.argtypes = [ctypes.c_int]
        _oracle = lib
    return _oracle


def ref_lib():
    global _ref
    if _ref is None:
        lib = _lib("libvpd_refharness.so")
        lib.vr_create.restype = ctypes.c_void_p
        lib.vr_create.argtypes = [ctypes.POINTER(VpdCase), ctypes.c_char_p]
        lib.vr_step.argtypes = [ctypes.c_void_p, ctypes.c_int32, _D]
        lib.vr_get.argtypes = [ctypes.c_void_p, ctypes.c_int32, _D]
        lib.vr_destroy.argtypes = [ctypes.c_void_p]
        lib.vr_num_points.restype = ctypes.c_int64
        lib.vr_num_points.argtypes = [ctypes.c_void_p]
        lib.vr_num_bonds.restype = ctypes.c_int64
        lib.vr_num_bonds.argtypes = [ctypes.c_void_p]
        lib.vr_neighbors.argtypes = [ctypes.c_void_p, _I64, _I32]
        lib.vr_stage_seconds.argtypes = [ctypes.c_void_p, _D]
        lib.vr_last_error.restype = ctypes.c_char_p
        lib.vr_build_neighbor_list.restype = ctypes.c_int64
        lib.vr_build_neighbor_list.argtypes = [_D, ctypes.c_int64, ctypes.c_double, _I64, _I32]
        _ref = lib
    return _ref


def reference_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libvpd_refharness.so"))


class _SimBase:
    _prefix = ""

    def __init__(self, case):
        self.case = case
        self.c_case = case.to_c()

    def _fn(self, name):
        return getattr(self._lib, self._prefix + name)

    @property
    def n_points(self):
        return int(self._fn("num_points")(self.h))

    @property
    def n_bonds(self):
        return int(self._fn("num_bonds")(self.h))

    def step(self, nsteps):
        diag = np.zeros((nsteps, DIAG_COLS))
        rc = self._fn("step")(self.h, nsteps, _dp(diag))
        if rc != 0:
            raise RuntimeError(f"{self._prefix}step failed with status {rc}")
        return diag

    def get(self, field):
        width = self.case.nstatev if field == "state" else FIELD_WIDTH[field]
        out = np.zeros((self.n_points, width))
        rc = self._fn("get")(self.h, FIELD[field], _dp(out))
        if rc != 0:
            raise RuntimeError(f"{self._prefix}get({field}) failed with status {rc}")
        return out

    def neighbors(self):
        row_ptr = np.zeros(self.n_points + 1, dtype=np.int64)
        col = np.zeros(max(self.n_bonds, 1), dtype=np.int32)
        self._fn("neighbors")(self.h, row_ptr.ctypes.data_as(_I64), col.ctypes.data_as(_I32))
        return row_ptr, col[: self.n_bonds]

    def close(self):
        if getattr(self, "h", None):
            self._fn("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OracleSim(_SimBase):
    """The C restatement's full increment (vo_create / vo_step / vo_get)."""
    _prefix = "vo_"

    def __init__(self, case, positions=None, volumes=None):
        super().__init__(case)
        self._lib = oracle_lib()
        status = ctypes.c_int(0)
        pos = None if positions is None else np.ascontiguousarray(positions, dtype=np.float64)
        vol = None if volumes is None else np.ascontiguousarray(volumes, dtype=np.float64)
        self.h = self._lib.vo_create(ctypes.byref(self.c_case),
                                     None if pos is None else _dp(pos),
                                     None if vol is None else _dp(vol), ctypes.byref(status))
        if not self.h:
            raise RuntimeError(f"vo_create failed with status {status.value}")


class RefSim(_SimBase):
    """The reference library's own modules driven in runMaterial's order."""
    _prefix = "vr_"

    def __init__(self, case, plugin="jc_vumat_plugin.so"):
        super().__init__(case)
        self._lib = ref_lib()
        self.h = self._lib.vr_create(ctypes.byref(self.c_case),
                                     os.path.join(REF_DIR, plugin).encode())
        if not self.h:
            raise RuntimeError("vr_create failed: " + self._lib.vr_last_error().decode())

    def stage_seconds(self):
        out = np.zeros(5)
        self._lib.vr_stage_seconds(self.h, _dp(out))
        return dict(zip(("deformation", "material", "damage", "force", "other"), out))


# ---------------------------------------------------------------- module functions
def neighbor_list(pos, horizon, reference=False):
    """Sorted neighbour CSR of points pos[n,3]: (row_ptr int64[n+1], col int32)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    n = pos.shape[0]
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    if reference:
        lib = ref_lib()
        total = lib.vr_build_neighbor_list(_dp(pos), n, horizon, row_ptr.ctypes.data_as(_I64),
                                           None)
        if total < 0:
            raise RuntimeError(lib.vr_last_error().decode())
        col = np.zeros(max(total, 1), dtype=np.int32)
        lib.vr_build_neighbor_list(_dp(pos), n, horizon, row_ptr.ctypes.data_as(_I64),
                                   col.ctypes.data_as(_I32))
        return row_ptr, col[:total]
    lib = oracle_lib()
    total = lib.vo_neighbor_count(_dp(pos), n, horizon, row_ptr.ctypes.data_as(_I64))
    if total < 0:
        raise RuntimeError(f"neighbour build failed with status {-total}")
    col = np.zeros(max(total, 1), dtype=np.int32)
    rc = lib.vo_neighbor_fill(_dp(pos), n, horizon, row_ptr.ctypes.data_as(_I64),
                              col.ctypes.data_as(_I32))
    if rc != 0:
        raise RuntimeError(f"neighbour fill failed with status {rc}")
    return row_ptr, col[:total]


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


def shape_inverse(pos, vol, row_ptr, col):
    pos, vol, row_ptr, col = _c(pos), _c(vol), _c(row_ptr, np.int64), _c(col, np.int32)
    out = np.zeros((pos.shape[0], 9))
    rc = oracle_lib().vo_shape_inverse(pos.shape[0], _dp(pos), _dp(vol),
                                       row_ptr.ctypes.data_as(_I64), col.ctypes.data_as(_I32),
                                       _dp(out))
    return rc, out


def deformation(pos, disp, vol, row_ptr, col, kinv):
    pos, disp, vol, kinv = _c(pos), _c(disp), _c(vol), _c(kinv)
    row_ptr, col = _c(row_ptr, np.int64), _c(col, np.int32)
    out = np.zeros((pos.shape[0], 9))
    oracle_lib().vo_deformation(pos.shape[0], _dp(pos), _dp(disp), _dp(vol),
                                row_ptr.ctypes.data_as(_I64), col.ctypes.data_as(_I32),
                                _dp(kinv), _dp(out))
    return out


def force(pos, vol, row_ptr, col, kinv, F, sigma, bond_damage=None):
    pos, vol, kinv, F, sigma = _c(pos), _c(vol), _c(kinv), _c(F), _c(sigma)
    row_ptr, col = _c(row_ptr, np.int64), _c(col, np.int32)
    bd = None if bond_damage is None else _c(bond_damage)
    out = np.zeros((pos.shape[0], 3))
    rc = oracle_lib().vo_force(pos.shape[0], _dp(pos), _dp(vol), row_ptr.ctypes.data_as(_I64),
                               col.ctypes.data_as(_I32), _dp(kinv), _dp(F), _dp(sigma),
                               None if bd is None else _dp(bd), _dp(out))
    return rc, out


def corotational(fN, fNP1, vN, rN, dt):
    fN, fNP1, vN, rN = _c(fN), _c(fNP1), _c(vN), _c(rN)
    n = fN.shape[0]
    outs = [np.zeros((n, 9)) for _ in range(5)]
    rc = oracle_lib().vo_corotational(n, _dp(fN), _dp(fNP1), _dp(vN), _dp(rN), dt,
                                      *[_dp(o) for o in outs])
    return rc, dict(zip(("rate_of_deformation", "relative_spin", "rotation", "left_stretch",
                         "strain"), outs))


def material_update(props, dt, F, state):
    """state: dict of arrays defgrad_old, left_stretch, rotation, strain,
    stress_corotational [n,9], state [n,nstatev], temperature, energy_internal,
    energy_inelastic [n]; updated copies are returned with stress_spatial."""
    s = {k: np.array(v, dtype=np.float64, copy=True) for k, v in state.items()}
    F = _c(F)
    n = F.shape[0]
    nstatev = s["state"].shape[1]
    props = _c(props)
    spatial = np.zeros((n, 9))
    rc = oracle_lib().vo_material_update(
        n, _dp(props), nstatev, dt, _dp(F), _dp(s["defgrad_old"]), _dp(s["left_stretch"]),
        _dp(s["rotation"]), _dp(s["strain"]), _dp(s["stress_corotational"]), _dp(s["state"]),
        _dp(s["temperature"]), _dp(s["energy_internal"]), _dp(s["energy_inelastic"]),
        _dp(spatial))
    s["stress_spatial"] = spatial
    return rc, s


def damage(pos, disp, vol, row_ptr, col, initiation, failure, bond_damage):
    pos, disp, vol = _c(pos), _c(disp), _c(vol)
    row_ptr, col = _c(row_ptr, np.int64), _c(col, np.int32)
    bd = np.array(bond_damage, dtype=np.float64, copy=True)
    idx = np.zeros(pos.shape[0])
    rc = oracle_lib().vo_damage(pos.shape[0], _dp(pos), _dp(disp), _dp(vol),
                                row_ptr.ctypes.data_as(_I64), col.ctypes.data_as(_I32),
                                initiation, failure, _dp(bd), _dp(idx))
    return rc, bd, idx


def set_perturbation(every):
    """Plants a one-ulp change in the deformation sum of every `every`-th point (0: none); for
    the sensitivity test only."""
    oracle_lib().vo_set_perturbation(int(every))


def jitter_value(seed, p, c, amp):
    return oracle_lib().vo_jitter_value(seed, p, c, amp)


def ramp(case, t):
    out = np.zeros(6)
    oracle_lib().vo_ramp(ctypes.byref(case.to_c()), t, _dp(out))
    return out


# ---------------------------------------------------------------- plugin ABI
def vumat_block(lib, props, dt, strain_inc, stress_old, state_old, temp_old, e_int_old,
                e_inel_old, nstatev=None, step_time=0.0, total_time=0.0):
    """Calls `vumat_adapter_call` of a loaded plugin (the restated JC in libvpd_oracle.so, or
    any library exporting the entry) on one block. Arrays are point-major [nblock, comps];
    they are packed to the plugin's column-major [comp][nblock] layout and back."""
    fn = lib.vumat_adapter_call
    nb = strain_inc.shape[0]
    nsv = nstatev or state_old.shape[1]
    ci = ctypes.c_int
    def col(a, comps):
        return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(nb, comps).T)
    inc, s_old, st_old = col(strain_inc, 6), col(stress_old, 6), col(state_old, nsv)
    t_old = np.ascontiguousarray(temp_old, dtype=np.float64).reshape(nb)
    ei_old = np.ascontiguousarray(e_int_old, dtype=np.float64).reshape(nb)
    ep_old = np.ascontiguousarray(e_inel_old, dtype=np.float64).reshape(nb)
    props = np.ascontiguousarray(props, dtype=np.float64)
    zeros = lambda *shape: np.zeros(shape)
    coord, char_len, dens = zeros(3, nb), np.ones(nb), np.full(nb, props[10])
    spin, stretch_old, defgrad_old, field_old = zeros(3, nb), zeros(6, nb), zeros(9, nb), zeros(1, nb)
    t_new, stretch_new, defgrad_new, field_new = zeros(nb), zeros(6, nb), zeros(9, nb), zeros(1, nb)
    s_new, st_new, ei_new, ep_new = zeros(6, nb), zeros(nsv, nb), zeros(nb), zeros(nb)
    cmname = ctypes.create_string_buffer(b" " * 80, 80)
    args = [ctypes.byref(ci(nb)), ctypes.byref(ci(3)), ctypes.byref(ci(3)), ctypes.byref(ci(nsv)),
            ctypes.byref(ci(1)), ctypes.byref(ci(len(props))), ctypes.byref(ci(0)),
            ctypes.byref(ctypes.c_double(step_time)), ctypes.byref(ctypes.c_double(total_time)),
            ctypes.byref(ctypes.c_double(dt)), cmname]
    arrays = [coord, char_len, props, dens, inc, spin, t_old, stretch_old, defgrad_old, field_old,
              s_old, st_old, ei_old, ep_old, t_new, stretch_new, defgrad_new, field_new, s_new,
              st_new, ei_new, ep_new]
    fn.restype = None
    fn(*args, *[_dp(a) for a in arrays])
    return {"stress": s_new.T.copy(), "state": st_new.T.copy(), "temperature": t_new,
            "energy_internal": ei_new, "energy_inelastic": ep_new}
