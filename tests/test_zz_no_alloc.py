"""vpd_force_density_noalloc, the entry point for hosts that cannot allocate device memory
during a step (their device memory belongs to their own pool, or their step loop cannot take
the device-wide synchronisation of cudaMalloc/cudaFree). Called through the C ABI, it must
give the same forces as vpd_force_density, on two calls in a row with different inputs (the
shared scratch keeps the previous call's contents), and reject blocks beyond its fixed
capacity. This file is collected last so a failure here leaves every other test already run."""
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
    case = tensile_bar(1, nx=14, ny=8, nz=7, jitter=0.05, jitter_seed=seed)
    sim = O.OracleSim(case)
    pos, vol = sim.get("position"), sim.get("volume")[:, 0]
    row_ptr, col = sim.neighbors()
    rng = np.random.default_rng(seed)
    n = len(vol)
    rc, kinv = O.shape_inverse(pos, vol, row_ptr, col)
    disp = 0.002 * rng.standard_normal(pos.shape)
    F = O.deformation(pos, disp, vol, row_ptr, col, kinv)
    s = rng.standard_normal((n, 3, 3)) * 150.0
    sigma = (s + s.transpose(0, 2, 1)).reshape(n, 9)
    bond = (rng.random(len(col)) < 0.05).astype(np.float64)
    return [cuda(pos), cuda(vol), cuda(row_ptr, torch.int64), cuda(col, torch.int32), cuda(kinv),
            cuda(F), cuda(sigma)], cuda(bond)


def test_noalloc_matches_allocating_entry_point_twice():
    for seed in (21, 22):  # two calls in a row on different inputs
        args, bond = block_inputs(seed)
        expected = vpd.force_density(*args, bond_damage=bond)
        out = torch.full_like(expected, float("nan"))
        vpd.force_density_noalloc(*args, out, bond_damage=bond)
        torch.cuda.synchronize()
        assert max_rel(out.cpu().numpy(), expected.cpu().numpy()) < 1e-12


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
