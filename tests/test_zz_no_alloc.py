"""vpd_force_density_noalloc, the entry point for hosts that cannot allocate device memory
during a step (their device memory belongs to their own pool, or their step loop cannot take
the device-wide synchronisation of cudaMalloc/cudaFree). Called through the C ABI, it must
give the same forces as vpd_force_density and as the oracle's force pass, on two calls in a
row with different inputs (the shared scratch keeps the previous call's contents); a call that
reports a singular deformation gradient must leave nothing behind that fails the next valid
call; blocks beyond its fixed capacity are rejected. This file is collected last so a failure
here leaves every other test already run."""
import numpy as np
import pytest

from conftest import max_rel

import oracle as O
import vpd
from vpd.case import tensile_bar

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def cuda(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(dtype=dtype, device="cuda").contiguous()


def block_inputs(seed):
    """A jittered 14x8x7 block with a random displacement, a symmetric stress and 5 % of the
    bonds broken; the host arrays and the oracle's forces for them."""
    case = tensile_bar(1, nx=14, ny=8, nz=7, jitter=0.05, jitter_seed=seed)
    sim = O.OracleSim(case)
    pos, vol = sim.get("position"), sim.get("volume")[:, 0]
    row_ptr, col = sim.neighbors()
    rng = np.random.default_rng(seed)
    n = len(vol)
    rc, kinv = O.shape_inverse(pos, vol, row_ptr, col)
    assert rc == 0
    disp = 0.002 * rng.standard_normal(pos.shape)
    F = O.deformation(pos, disp, vol, row_ptr, col, kinv)
    s = rng.standard_normal((n, 3, 3)) * 150.0
    sigma = (s + s.transpose(0, 2, 1)).reshape(n, 9)
    bond = (rng.random(len(col)) < 0.05).astype(np.float64)
    rc, f_oracle = O.force(pos, vol, row_ptr, col, kinv, F, sigma, bond)
    assert rc == 0
    host = dict(pos=pos, vol=vol, row_ptr=row_ptr, col=col, kinv=kinv, F=F, sigma=sigma, bond=bond)
    return host, f_oracle


def device_args(h, F=None):
    return [cuda(h["pos"]), cuda(h["vol"]), cuda(h["row_ptr"], torch.int64),
            cuda(h["col"], torch.int32), cuda(h["kinv"]), cuda(h["F"] if F is None else F),
            cuda(h["sigma"])]


def test_noalloc_matches_allocating_entry_point_and_oracle_twice():
    for seed in (21, 22):  # two calls in a row on different inputs
        h, f_oracle = block_inputs(seed)
        args, bond = device_args(h), cuda(h["bond"])
        expected = vpd.force_density(*args, bond_damage=bond)
        out = torch.full_like(expected, float("nan"))
        vpd.force_density_noalloc(*args, out, bond_damage=bond)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert max_rel(got, expected.cpu().numpy()) < 1e-12
        assert max_rel(got, f_oracle) < 1e-12


def test_noalloc_singular_call_then_valid_call():
    """A call whose deformation gradient is singular at one point reports VPD_ERR_SINGULAR, as
    vpd_force_density does; the status word lives in the shared scratch, so the next valid
    call must come back clean and match the oracle."""
    h, f_oracle = block_inputs(23)
    F_bad = h["F"].copy()
    F_bad[5] = 0.0
    out = torch.zeros((len(h["vol"]), 3), dtype=torch.float64, device="cuda")
    with pytest.raises(vpd.VpdError) as e:
        vpd.force_density_noalloc(*device_args(h, F_bad), out, bond_damage=cuda(h["bond"]))
    assert e.value.status == 3
    with pytest.raises(vpd.VpdError) as e:
        vpd.force_density(*device_args(h, F_bad), bond_damage=cuda(h["bond"]))
    assert e.value.status == 3
    out = torch.full((len(h["vol"]), 3), float("nan"), dtype=torch.float64, device="cuda")
    vpd.force_density_noalloc(*device_args(h), out, bond_damage=cuda(h["bond"]))
    torch.cuda.synchronize()
    assert max_rel(out.cpu().numpy(), f_oracle) < 1e-12


def test_noalloc_rejects_blocks_beyond_capacity():
    n = 65537
    pos = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    vol = torch.ones(n, dtype=torch.float64, device="cuda")
    row_ptr = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    col = torch.zeros(1, dtype=torch.int32, device="cuda")
    t9 = torch.zeros((n, 9), dtype=torch.float64, device="cuda")
    out = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(vpd.VpdError) as e:
        vpd.force_density_noalloc(pos, vol, row_ptr, col, t9, t9, t9, out)
    assert e.value.status == 5 and "65536" in str(e.value)
