"""Python binding of libvpd_gpu.so, the B200 correspondence-PD increment.

Mirrors the reference's host interface for the PD path:

  * ``Simulation`` -- runMaterial of src/host/BoundaryValueCaseRunner.cpp:139-337 on the GPU:
    ``step(n)`` returns the timeseries rows (the numeric columns of timeseries.csv),
    ``field(name)`` the per-node state (writeSnapshot, MaterialState, ExplicitDynamicState),
    ``neighbors()`` the sorted neighbour lists (ParticleBlock::neighbors) as CSR;
  * module functions taking torch CUDA tensors -- ``build_neighbor_list``
    (buildNeighborList), ``shape_tensor_inverse`` (PdCorrespondenceSkeleton::initialize),
    ``deformation_gradients``, ``force_density``, ``corotational_update``,
    ``material_update`` (VumatPdCorrespondenceMaterial::update with the Johnson-Cook VUMAT),
    ``damage_update`` (PdSimpleDamage::update, critical_stretch);
  * ``vumat_adapter_call`` -- the plugin entry the reference's VumatMaterialAdapter dlopens.

Errors raise ``VpdError`` carrying the library's status and message, as the reference
throws std::runtime_error. There is no CPU fallback: without the built library (``make -C
vumat-pd_b200``) or without a CUDA device every call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .case import (DIAG, DIAG_COLUMNS, FIELD, FIELD_WIDTH, FIELDS, Case, VpdCase, pd_coarse,
                   stable_dt, steel_props, tensile_bar)

__all__ = ["Simulation", "VpdError", "Case", "pd_coarse", "tensile_bar", "stable_dt",
           "steel_props", "DIAG", "DIAG_COLUMNS", "FIELDS", "library", "library_path"]

LIB_NAME = "libvpd_gpu.so"
_HERE = os.path.dirname(os.path.abspath(__file__))


def library_path() -> str:
    return os.path.join(os.path.dirname(_HERE), LIB_NAME)


class VpdError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[vpd status {status}] {message}")
        self.status = status


_D = ctypes.POINTER(ctypes.c_double)
_I64 = ctypes.POINTER(ctypes.c_int64)
_I32 = ctypes.POINTER(ctypes.c_int32)
_VP = ctypes.c_void_p
_lib = None


def library():
    """Loads libvpd_gpu.so once; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise VpdError(-1, f"{path} is missing; build it with `make -C vumat-pd_b200`")
    lib = ctypes.CDLL(path)
    lib.vpd_abi_version.restype = ctypes.c_int
    lib.vpd_last_error.restype = ctypes.c_char_p
    lib.vpd_create.argtypes = [ctypes.POINTER(VpdCase), _D, _D, ctypes.POINTER(_VP)]
    lib.vpd_destroy.argtypes = [_VP]
    lib.vpd_num_points.restype = ctypes.c_int64
    lib.vpd_num_points.argtypes = [_VP]
    lib.vpd_num_bonds.restype = ctypes.c_int64
    lib.vpd_num_bonds.argtypes = [_VP]
    lib.vpd_bond_layout_words.argtypes = [_VP]
    lib.vpd_step.argtypes = [_VP, ctypes.c_int32, _D]
    lib.vpd_download.argtypes = [_VP, ctypes.c_int32, _D]
    lib.vpd_neighbors.argtypes = [_VP, _I64, _I32]
    lib.vpd_stream.restype = _VP
    lib.vpd_stream.argtypes = [_VP]
    lib.vpd_last_step_ms.argtypes = [_VP, _D]
    lib.vpd_profile_increment.argtypes = [_VP, ctypes.c_int32, _D]
    lib.vpd_field_width.argtypes = [_VP, ctypes.c_int]
    lib.vpd_build_neighbor_list.argtypes = [_VP, ctypes.c_int64, ctypes.c_double, _VP, _VP, _I64, _VP]
    lib.vpd_shape_tensor_inverse.argtypes = [_VP, _VP, ctypes.c_int64, _VP, _VP, _VP, _VP]
    lib.vpd_deformation_gradients.argtypes = [_VP, _VP, _VP, ctypes.c_int64, _VP, _VP, _VP, _VP, _VP]
    lib.vpd_force_density.argtypes = [_VP, _VP, ctypes.c_int64, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]
    lib.vpd_force_density_noalloc.argtypes = [_VP, _VP, ctypes.c_int64, _VP, _VP, _VP, _VP, _VP,
                                              _VP, _VP, _VP]
    lib.vpd_corotational_update.argtypes = [ctypes.c_int64, _VP, _VP, _VP, _VP, ctypes.c_double,
                                            _VP, _VP, _VP, _VP, _VP, _VP]
    lib.vpd_material_update.argtypes = [ctypes.c_int64, _D, ctypes.c_int32, ctypes.c_double] + [_VP] * 12
    lib.vpd_jc_return_map.argtypes = [ctypes.c_int64, _D, ctypes.c_double, _VP, _VP, _VP, ctypes.c_int32,
                                      ctypes.c_int32, _VP, _VP, _VP, _VP]
    lib.vpd_damage_update.argtypes = [_VP, _VP, _VP, ctypes.c_int64, _VP, _VP, ctypes.c_double,
                                      ctypes.c_double, _VP, _VP, _VP]
    lib.vpd_mlp_forward.argtypes = [_VP, _VP, _VP, ctypes.c_int64, _VP, _VP]
    lib.vpd_surrogate_samples.argtypes = [_D, ctypes.c_uint64, ctypes.c_int64, _VP, _VP, _VP]
    lib.vpd_train_surrogate.argtypes = [ctypes.POINTER(SurrogateConfig), _VP, _VP,
                                        ctypes.POINTER(SurrogateReport)]
    lib.vpd_set_surrogate.argtypes = [_VP, _VP, _VP, ctypes.c_int32, ctypes.c_int32]
    lib.vpd_mlp_gradients.argtypes = [_VP, _VP, _VP, _VP, ctypes.c_int64, _VP, _VP]
    lib.vpd_set_initial_state.argtypes = [_VP, _VP, ctypes.c_int32]
    lib.vpd_set_internal_indicator.argtypes = [_VP, _VP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
    lib.vpd_checkpoint_bytes.argtypes = [_VP]
    lib.vpd_checkpoint_bytes.restype = ctypes.c_int64
    lib.vpd_checkpoint_save.argtypes = [_VP, _VP, ctypes.c_int64]
    lib.vpd_checkpoint_load.argtypes = [_VP, _VP, ctypes.c_int64]
    lib.vpd_set_host_vumat.argtypes = [_VP, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _VP,
                                       ctypes.c_int32, ctypes.c_int32, ctypes.c_double]
    _lib = lib
    return lib


def _check(rc: int):
    if rc != 0:
        raise VpdError(rc, library().vpd_last_error().decode(errors="replace"))


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_D)


MAX_EPOCHS = 64
SAMPLE_RECORD = 26
GUESS = {"network": 0, "warm_start": 1, "hybrid": 2}


class SurrogateConfig(ctypes.Structure):
    _fields_ = [("props", ctypes.c_double * 14), ("samples", ctypes.c_int64),
                ("epochs", ctypes.c_int32), ("batch", ctypes.c_int32),
                ("learning_rate", ctypes.c_double), ("seed", ctypes.c_uint64),
                ("validation_fraction", ctypes.c_double)]


class SurrogateReport(ctypes.Structure):
    _fields_ = [("epochs_run", ctypes.c_int32), ("epoch_loss", ctypes.c_double * MAX_EPOCHS),
                ("validation_loss", ctypes.c_double), ("ratio_rmse", ctypes.c_double),
                ("stress_rmse", ctypes.c_double), ("plastic_fraction", ctypes.c_double),
                ("train_ms", ctypes.c_double)]


def surrogate_samples(props, seed: int, count: int, records: bool = False):
    """Increments solved by the device VUMAT: (features [count,16], targets [count,16],
    records [count, SAMPLE_RECORD] or None), float32 / float64 numpy arrays."""
    props = np.ascontiguousarray(props, dtype=np.float64)
    f = np.zeros((count, 16), dtype=np.float32)
    t = np.zeros((count, 16), dtype=np.float32)
    r = np.zeros((count, SAMPLE_RECORD)) if records else None
    _check(library().vpd_surrogate_samples(_dp(props), seed, count, f.ctypes.data_as(_VP),
                                           t.ctypes.data_as(_VP),
                                           None if r is None else r.ctypes.data_as(_VP)))
    return f, t, r


def train_surrogate(props, samples: int = 2_000_000, epochs: int = 20, batch: int = 8192,
                    learning_rate: float = 1e-3, seed: int = 2026, validation_fraction: float = 0.05):
    """Trains the Johnson-Cook surrogate on the GPU. Returns (weights uint16 [VPD_MLP_WEIGHTS],
    biases float32 [400], report dict)."""
    cfg = SurrogateConfig()
    for k, v in enumerate(props):
        cfg.props[k] = float(v)
    cfg.samples, cfg.epochs, cfg.batch = samples, epochs, batch
    cfg.learning_rate, cfg.seed, cfg.validation_fraction = learning_rate, seed, validation_fraction
    w = np.zeros(MLP_WEIGHTS, dtype=np.uint16)
    b = np.zeros(MLP_PARAMS - MLP_WEIGHTS, dtype=np.float32)
    rep = SurrogateReport()
    _check(library().vpd_train_surrogate(ctypes.byref(cfg), w.ctypes.data_as(_VP),
                                         b.ctypes.data_as(_VP), ctypes.byref(rep)))
    report = {"epoch_loss": [rep.epoch_loss[e] for e in range(rep.epochs_run)],
              "validation_loss": rep.validation_loss, "ratio_rmse": rep.ratio_rmse,
              "stress_rmse": rep.stress_rmse, "plastic_fraction": rep.plastic_fraction,
              "train_ms": rep.train_ms}
    return w, b, report


class Simulation:
    """One regional boundary-value case on the GPU (a vpd_handle)."""

    def __init__(self, case: Case, positions=None, volumes=None):
        lib = library()
        self.case = case
        self._c = case.to_c()
        h = _VP()
        pos = None if positions is None else np.ascontiguousarray(positions, dtype=np.float64)
        vol = None if volumes is None else np.ascontiguousarray(volumes, dtype=np.float64)
        _check(lib.vpd_create(ctypes.byref(self._c), None if pos is None else _dp(pos),
                              None if vol is None else _dp(vol), ctypes.byref(h)))
        self._h = h

    @property
    def n_points(self) -> int:
        return int(library().vpd_num_points(self._h))

    @property
    def n_bonds(self) -> int:
        return int(library().vpd_num_bonds(self._h))

    @property
    def layout_words(self) -> int:
        """Lattice-stencil mask words per point (0: sliced-ELL index layout)."""
        return int(library().vpd_bond_layout_words(self._h))

    def step(self, nsteps: int, diagnostics: bool = True) -> np.ndarray | None:
        """Advances nsteps increments; returns nsteps x len(DIAG_COLUMNS) timeseries rows."""
        rows = np.zeros((nsteps, len(DIAG_COLUMNS))) if diagnostics else None
        _check(library().vpd_step(self._h, nsteps, _dp(rows) if diagnostics else None))
        return rows

    def set_surrogate(self, weights=None, biases=None, guess: str = "network",
                      newton_steps: int = 2):
        """Attaches the learned return map (material_mode MATERIAL_SURROGATE cases)."""
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.uint16)
        b = None if biases is None else np.ascontiguousarray(biases, dtype=np.float32)
        _check(library().vpd_set_surrogate(self._h, None if w is None else w.ctypes.data_as(_VP),
                                           None if b is None else b.ctypes.data_as(_VP),
                                           GUESS[guess], newton_steps))

    def set_host_vumat(self, plugin_path: str, props, nstatev: int, density: float,
                       cmname: str = "JOHNSONCOOK", symbol: str = "vumat_adapter_call"):
        """Runs the material update through a host VUMAT plugin (a shared library exporting the
        reference's vumat_adapter_call ABI) instead of the device Johnson-Cook update; the
        rest of each increment stays on the GPU. Call before the first step."""
        pr = np.ascontiguousarray(props, dtype=np.float64)
        _check(library().vpd_set_host_vumat(self._h, os.fsencode(plugin_path), symbol.encode(),
                                            cmname.encode(), pr.ctypes.data_as(_VP), pr.size,
                                            nstatev, density))

    def set_initial_state(self, state):
        """Every point's VUMAT state before the first step (vpd_set_initial_state)."""
        st = np.ascontiguousarray(state, dtype=np.float64)
        _check(library().vpd_set_initial_state(self._h, st.ctypes.data_as(_VP), st.size))

    def set_internal_indicator(self, indices, reduction: str = "max", transform: str = "identity"):
        """The diagnostics' internal indicator (vpd_set_internal_indicator)."""
        idx = np.ascontiguousarray(indices, dtype=np.int32)
        _check(library().vpd_set_internal_indicator(self._h, idx.ctypes.data_as(_VP), idx.size,
                                                    int(reduction == "min"), int(transform == "one_minus")))

    def checkpoint(self) -> bytes:
        """The state this simulation carries into its next increment (vpd_checkpoint_save)."""
        lib = library()
        size = lib.vpd_checkpoint_bytes(self._h)
        buf = ctypes.create_string_buffer(size)
        _check(lib.vpd_checkpoint_save(self._h, buf, size))
        return buf.raw

    def restore(self, data: bytes):
        """Continues from a checkpoint of a simulation of the same case (vpd_checkpoint_load)."""
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        _check(library().vpd_checkpoint_load(self._h, buf, len(data)))

    def last_step_ms(self) -> float:
        out = ctypes.c_double()
        _check(library().vpd_last_step_ms(self._h, ctypes.byref(out)))
        return out.value

    def profile_stages(self, nsteps: int) -> dict:
        """Advances nsteps increments with CUDA events between the kernels; mean ms each."""
        out = np.zeros(4)
        _check(library().vpd_profile_increment(self._h, nsteps, _dp(out)))
        return dict(zip(("deformation", "material", "force", "integrate"), out.tolist()))

    def field(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        width = self.case.nstatev if name == "state" else FIELD_WIDTH[name]
        if out is None:
            out = np.empty((self.n_points, width))
        _check(library().vpd_download(self._h, FIELD[name], _dp(out)))
        return out

    def neighbors(self):
        row_ptr = np.zeros(self.n_points + 1, dtype=np.int64)
        col = np.zeros(max(self.n_bonds, 1), dtype=np.int32)
        _check(library().vpd_neighbors(self._h, row_ptr.ctypes.data_as(_I64),
                                       col.ctypes.data_as(_I32)))
        return row_ptr, col[: self.n_bonds]

    def stream(self) -> int:
        return int(library().vpd_stream(self._h) or 0)

    def close(self):
        if getattr(self, "_h", None):
            library().vpd_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- module functions
def _ptr(t):
    if t is None:
        return None
    if not (t.is_cuda and t.is_contiguous()):
        raise ValueError("module functions take contiguous CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def build_neighbor_list(positions, horizon: float):
    """buildNeighborList on a CUDA float64 tensor [n,3] -> (row_ptr int64[n+1], col int32)."""
    import torch
    n = positions.shape[0]
    row_ptr = torch.empty(n + 1, dtype=torch.int64, device=positions.device)
    total = ctypes.c_int64()
    lib = library()
    _check(lib.vpd_build_neighbor_list(_ptr(positions), n, horizon, _ptr(row_ptr), None,
                                       ctypes.byref(total), _stream()))
    col = torch.empty(max(total.value, 1), dtype=torch.int32, device=positions.device)
    _check(lib.vpd_build_neighbor_list(_ptr(positions), n, horizon, _ptr(row_ptr), _ptr(col),
                                       ctypes.byref(total), _stream()))
    return row_ptr, col[: total.value]


def shape_tensor_inverse(positions, volumes, row_ptr, col):
    import torch
    out = torch.empty((positions.shape[0], 9), dtype=torch.float64, device=positions.device)
    _check(library().vpd_shape_tensor_inverse(_ptr(positions), _ptr(volumes), positions.shape[0],
                                              _ptr(row_ptr), _ptr(col), _ptr(out), _stream()))
    return out


def deformation_gradients(positions, displacement, volumes, row_ptr, col, kinv):
    import torch
    out = torch.empty((positions.shape[0], 9), dtype=torch.float64, device=positions.device)
    _check(library().vpd_deformation_gradients(_ptr(positions), _ptr(displacement), _ptr(volumes),
                                               positions.shape[0], _ptr(row_ptr), _ptr(col),
                                               _ptr(kinv), _ptr(out), _stream()))
    return out


def force_density(positions, volumes, row_ptr, col, kinv, defgrad, stress, bond_damage=None):
    import torch
    out = torch.empty((positions.shape[0], 3), dtype=torch.float64, device=positions.device)
    _check(library().vpd_force_density(_ptr(positions), _ptr(volumes), positions.shape[0],
                                       _ptr(row_ptr), _ptr(col), _ptr(kinv), _ptr(defgrad),
                                       _ptr(stress), _ptr(bond_damage), _ptr(out), _stream()))
    return out


def force_density_noalloc(positions, volumes, row_ptr, col, kinv, defgrad, stress, out,
                          bond_damage=None):
    """force_density for callers that cannot allocate device memory: the library allocates
    nothing (its scratch is a fixed array, at most 65536 points per call) and writes into the
    caller's ``out`` [n,3]. Calls that overlap on the GPU share that scratch and race."""
    _check(library().vpd_force_density_noalloc(_ptr(positions), _ptr(volumes), positions.shape[0],
                                               _ptr(row_ptr), _ptr(col), _ptr(kinv),
                                               _ptr(defgrad), _ptr(stress), _ptr(bond_damage),
                                               _ptr(out), _stream()))
    return out


def corotational_update(defgrad_old, defgrad_new, stretch_old, rotation_old, dt):
    import torch
    n = defgrad_old.shape[0]
    outs = [torch.empty((n, 9), dtype=torch.float64, device=defgrad_old.device) for _ in range(5)]
    _check(library().vpd_corotational_update(n, _ptr(defgrad_old), _ptr(defgrad_new),
                                             _ptr(stretch_old), _ptr(rotation_old), dt,
                                             *[_ptr(o) for o in outs], _stream()))
    return dict(zip(("rate_of_deformation", "relative_spin", "rotation", "left_stretch",
                     "strain"), outs))


def material_update(props, dt, defgrad_new, state):
    """state: dict of CUDA tensors updated in place (defgrad_old, left_stretch, rotation,
    strain, stress_corotational [n,9]; state [n,nstatev]; temperature, energy_internal,
    energy_inelastic [n]). Returns the spatial stress [n,9]."""
    import torch
    n = defgrad_new.shape[0]
    props_np = np.ascontiguousarray(props, dtype=np.float64)
    spatial = torch.empty((n, 9), dtype=torch.float64, device=defgrad_new.device)
    s = state
    _check(library().vpd_material_update(
        n, _dp(props_np), s["state"].shape[1], dt, _ptr(defgrad_new), _ptr(s["defgrad_old"]),
        _ptr(s["left_stretch"]), _ptr(s["rotation"]), _ptr(s["strain"]),
        _ptr(s["stress_corotational"]), _ptr(s["state"]), _ptr(s["temperature"]),
        _ptr(s["energy_internal"]), _ptr(s["energy_inelastic"]), _ptr(spatial), _stream()))
    return spatial


def jc_return_map(props, dt, strain_inc, stress, state, method=0):
    """The Johnson-Cook return map alone on CUDA tensors: strain_inc, stress [n,6], state
    [n,nstatev] (float64) -> (ep_inc, yield, iterations) [n]. method 0: the certified bisection of
    the increment kernels; 1: the literal bisection (the same bits)."""
    import torch
    n = strain_inc.shape[0]
    props_np = np.ascontiguousarray(props, dtype=np.float64)
    dev = strain_inc.device
    ep = torch.empty(n, dtype=torch.float64, device=dev)
    y = torch.empty(n, dtype=torch.float64, device=dev)
    it = torch.empty(n, dtype=torch.int32, device=dev)
    _check(library().vpd_jc_return_map(n, _dp(props_np), dt, _ptr(strain_inc), _ptr(stress), _ptr(state),
                                       state.shape[1], method, _ptr(ep), _ptr(y), _ptr(it), _stream()))
    return ep, y, it


def mlp_forward(weight_bits, biases, x):
    """Surrogate network forward on the tensor cores: weight_bits int16/uint16 CUDA tensor
    [VPD_MLP_WEIGHTS] (bf16 bit patterns), biases float32 [400], x float32 [B,16] -> [B,16]."""
    import torch
    out = torch.empty((x.shape[0], 16), dtype=torch.float32, device=x.device)
    _check(library().vpd_mlp_forward(_ptr(weight_bits), _ptr(biases), _ptr(x), x.shape[0],
                                     _ptr(out), _stream()))
    return out


def mlp_gradients(weight_bits, biases, x, gout):
    """d/dparams of sum(network(x) * gout) -> float32 [VPD_MLP_PARAMS] (weights, then biases)."""
    import torch
    grad = torch.empty(MLP_PARAMS, dtype=torch.float32, device=x.device)
    _check(library().vpd_mlp_gradients(_ptr(weight_bits), _ptr(biases), _ptr(x), _ptr(gout),
                                       x.shape[0], _ptr(grad), _stream()))
    return grad


MLP_WEIGHTS = 36864
MLP_PARAMS = 37264


def damage_update(positions, displacement, volumes, row_ptr, col, initiation, failure,
                  bond_damage):
    import torch
    idx = torch.empty(positions.shape[0], dtype=torch.float64, device=positions.device)
    _check(library().vpd_damage_update(_ptr(positions), _ptr(displacement), _ptr(volumes),
                                       positions.shape[0], _ptr(row_ptr), _ptr(col), initiation,
                                       failure, _ptr(bond_damage), _ptr(idx), _stream()))
    return idx
