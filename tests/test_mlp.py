"""Surrogate network: the tcgen05 forward/backward kernels against the CPU FP64 network.

CPU tests pin the oracle network itself (finite differences, BF16 rounding). GPU tests call
vpd_mlp_forward / vpd_mlp_gradients through the C ABI and compare with
  * the oracle with BF16 rounding emulated at the device's storage points (tolerance 2e-3 of
    the result's norm: the remaining difference is FP32 accumulation order, __expf, and rare
    BF16 rounding flips of activations), and
  * the plain FP64 network (tolerance 3e-2 of the norm: what BF16 storage costs).
"""
import numpy as np
import pytest

import mlp as M

torch = pytest.importorskip("torch")


def rel(a, ref):
    a, ref = np.asarray(a, np.float64), np.asarray(ref, np.float64)
    return float(np.linalg.norm(a - ref) / max(np.linalg.norm(ref), 1e-300))


def inputs(batch, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((batch, M.IN)).astype(np.float32)
    g = (rng.standard_normal((batch, M.OUT)) / batch).astype(np.float32)
    return x, g


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -3.140625, 1e-3, 65504.0])
    r = M.round_bf16(vals)
    assert r[0] == 1.0
    assert r[1] == 1.0                       # tie -> even
    assert r[2] == 1.0 + 2 * 2.0 ** -7       # tie -> even (up)
    assert r[3] == -3.140625
    assert abs(r[4] - 1e-3) / 1e-3 < 2 ** -8
    assert M.bf16_bits(np.float32(1.0)) == 0x3F80


def test_oracle_gradient_matches_finite_differences():
    w, b = M.init_params(3, zero_padding=False)
    x, g = inputs(37, 4)
    grad = M.gradients(w, b, x, g, emulate_bf16=False)
    for idx in (0, 77, 200, 300, 390, 399):
        fd = M.loss_and_grad_fd(w, b, x, g, idx)
        assert abs(grad[M.N_WEIGHTS + idx] - fd) <= 1e-7 * max(1.0, abs(fd))
    # a weight: perturb by exactly one bf16 step around a representable value
    wv = M.bf16_value(w)
    k = 2048 + 5 * 128 + 17
    out0 = np.sum(M.forward(w, b, x, emulate_bf16=False) * g)
    w2 = w.copy()
    w2[k] = M.bf16_bits(np.float32(wv[k] * (1 + 2.0 ** -7)))[()]
    out1 = np.sum(M.forward(w2, b, x, emulate_bf16=False) * g)
    dw = M.bf16_value(w2[k]) - wv[k]
    assert abs((out1 - out0) / dw - grad[k]) <= 2e-2 * max(abs(grad[k]), 1e-3)


def test_bf16_emulation_close_to_fp64():
    w, b = M.init_params(5)
    x, g = inputs(512, 6)
    assert rel(M.forward(w, b, x), M.forward(w, b, x, emulate_bf16=False)) < 1e-2
    assert rel(M.gradients(w, b, x, g), M.gradients(w, b, x, g, emulate_bf16=False)) < 3e-2


# ------------------------------------------------------------------ device kernels
def dev(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype).contiguous()


def dev_params(w, b):
    return dev(w.view(np.int16), torch.int16), dev(b, torch.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [1, 128, 1000, 8192])
def test_forward_matches_oracle(batch):
    import vpd
    w, b = M.init_params(11, zero_padding=False)
    x, _ = inputs(batch, 12)
    wd, bd = dev_params(w, b)
    out = vpd.mlp_forward(wd, bd, dev(x, torch.float32)).cpu().numpy()
    assert rel(out, M.forward(w, b, x)) < 2e-3
    assert rel(out, M.forward(w, b, x, emulate_bf16=False)) < 3e-2


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [1, 200, 4096])
def test_gradients_match_oracle(batch):
    import vpd
    w, b = M.init_params(21, zero_padding=False)
    x, g = inputs(batch, 22)
    wd, bd = dev_params(w, b)
    grad = vpd.mlp_gradients(wd, bd, dev(x, torch.float32), dev(g, torch.float32)).cpu().numpy()
    ref = M.gradients(w, b, x, g)
    ref64 = M.gradients(w, b, x, g, emulate_bf16=False)
    # per parameter block, so a wrong layer cannot hide behind a large one
    bounds = np.cumsum([0] + [r * c for r, c in M.SHAPES] + [128, 128, 128, 16])
    for lo, hi in zip(bounds[:-1], bounds[1:]):
        assert rel(grad[lo:hi], ref[lo:hi]) < 2e-3, (lo, hi)
        assert rel(grad[lo:hi], ref64[lo:hi]) < 3e-2, (lo, hi)


@pytest.mark.gpu
def test_forward_rejects_bad_arguments():
    import vpd
    w, b = M.init_params(1)
    wd, bd = dev_params(w, b)
    x = torch.zeros((0, 16), dtype=torch.float32, device="cuda")
    with pytest.raises(vpd.VpdError):
        vpd.mlp_forward(wd, bd, x)
