"""ORACLE / TEST INFRASTRUCTURE ONLY -- CPU FP64 restatement of the surrogate network.

The surrogate (10 -> 128 -> 128 -> 128 -> 7, SiLU) has no counterpart in the reference; this
file is the checker for the tensor-core kernels behind ``vpd_mlp_forward`` and
``vpd_mlp_gradients``. Parameter layout is the library's flat order: w1 [128][16],
w2 [128][128], w3 [128][128], w4 [16][128] (row-major [out][in]), then b1, b2, b3 [128], b4 [16].

``emulate_bf16=True`` rounds to bfloat16 (round to nearest even) exactly where the device
kernels store BF16 operands: the inputs, each hidden activation, and each layer's dZ before
the weight-gradient and input-gradient products. Everything else is FP64. With
``emulate_bf16=False`` the same network runs in plain FP64 (weights still the BF16 values),
which is the mathematical gradient the device result approximates.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 16, 128, 16
SHAPES = [(HID, IN), (HID, HID), (HID, HID), (OUT, HID)]
N_WEIGHTS = sum(a * b for a, b in SHAPES)            # 36864
N_PARAMS = N_WEIGHTS + 3 * HID + OUT                   # 37264


def bf16_bits(a) -> np.ndarray:
    """float -> bfloat16 bit patterns (uint16), round to nearest even (NaN not handled)."""
    f = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    rounded = (f + 0x7FFF + ((f >> 16) & 1)) >> 16
    return rounded.astype(np.uint16)


def bf16_value(bits) -> np.ndarray:
    return (np.asarray(bits, dtype=np.uint32) << 16).view(np.float32).astype(np.float64)


def round_bf16(a) -> np.ndarray:
    return bf16_value(bf16_bits(a)).reshape(np.shape(a))


def unpack(weight_bits, biases):
    """Flat (uint16 weights, float biases) -> lists of FP64 matrices and bias vectors."""
    w = bf16_value(weight_bits)
    mats, off = [], 0
    for r, c in SHAPES:
        mats.append(w[off:off + r * c].reshape(r, c))
        off += r * c
    b = np.asarray(biases, dtype=np.float64)
    bs = [b[0:128], b[128:256], b[256:384], b[384:400]]
    return mats, bs


def init_params(seed: int, zero_padding: bool = True, features: int = 10, targets: int = 7):
    """Random weights (bf16 bits) ~ N(0, 1/fan_in) and small random biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for r, c in SHAPES:
        m = rng.standard_normal((r, c)) / np.sqrt(c)
        parts.append(m)
    if zero_padding:
        parts[0][:, features:] = 0.0
        parts[3][targets:, :] = 0.0
    wbits = bf16_bits(np.concatenate([p.ravel() for p in parts]))
    biases = (0.1 * rng.standard_normal(3 * HID + OUT)).astype(np.float32)
    if zero_padding:
        biases[384 + targets:] = 0.0
    return wbits, biases


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(weight_bits, biases, x, emulate_bf16=True, keep=False):
    """out [B][16]; with keep=True also returns the saved (inputs, pre-activations, activations)."""
    rnd = round_bf16 if emulate_bf16 else (lambda a: a)
    (w1, w2, w3, w4), (b1, b2, b3, b4) = unpack(weight_bits, biases)
    y0 = rnd(np.asarray(x, dtype=np.float64))
    zs, ys = [], [y0]
    y = y0
    for w, b in ((w1, b1), (w2, b2), (w3, b3)):
        z = y @ w.T + b
        y = rnd(_silu(z))
        zs.append(z)
        ys.append(y)
    out = y @ w4.T + b4
    return (out, zs, ys) if keep else out


def gradients(weight_bits, biases, x, gout, emulate_bf16=True):
    """d/dparams of sum(out * gout): flat [N_PARAMS] (weights then biases), FP64."""
    rnd = round_bf16 if emulate_bf16 else (lambda a: a)
    (w1, w2, w3, w4), _ = unpack(weight_bits, biases)
    _, zs, ys = forward(weight_bits, biases, x, emulate_bf16, keep=True)
    dz = np.asarray(gout, dtype=np.float64)
    gw, gb = [None] * 4, [None] * 4
    dzb = rnd(dz)
    gw[3] = dzb.T @ ys[3]
    gb[3] = dz.sum(axis=0)
    dy = dzb @ w4
    for layer, w in ((2, w3), (1, w2), (0, w1)):
        dz = dy * _silu_grad(zs[layer])
        dzb = rnd(dz)
        gw[layer] = dzb.T @ ys[layer]
        gb[layer] = dz.sum(axis=0)
        dy = dzb @ w
    return np.concatenate([g.ravel() for g in gw] + [g.ravel() for g in gb])


def loss_and_grad_fd(weight_bits, biases, x, gout, index, h=1e-3):
    """Central finite difference of sum(out * gout) in bias `index` (a bias is FP32 on the
    device, so it can be perturbed without BF16 rounding); plain FP64 network."""
    b = np.asarray(biases, dtype=np.float64).copy()
    b[index] += h
    fp = np.sum(forward(weight_bits, b, x, emulate_bf16=False) * gout)
    b[index] -= 2 * h
    fm = np.sum(forward(weight_bits, b, x, emulate_bf16=False) * gout)
    return (fp - fm) / (2 * h)
