"""Parity of the CUDA path (through the C ABI) with the oracle, the reference library's
fixtures and the reference's archived run. Tolerances: neighbour lists bit-exact; FP64
fields and timeseries within the stated relative tolerances; stress history NRMSE <= 1e-6."""
import numpy as np
import pytest

from conftest import golden, load_golden_timeseries, max_rel, nrmse

import oracle as O
import vpd
from vpd.case import PRECISION_FP64, REFERENCE_JC_PROPS, Case, pd_coarse, tensile_bar

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

STRESS = vpd.DIAG["average_axial_stress_MPa"]


def cuda(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(dtype=dtype, device="cuda").contiguous()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


# ---------------------------------------------------------------- neighbour lists
def test_neighbor_lattice_regression():
    n = 9
    ijk = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 3)
    d2 = ((ijk[:, None, :] - ijk[None, :, :]) ** 2).sum(-1)
    for h in (2.0 / 3.0, 1.0, 2.0):
        for shift in (0.0, -123.456, 10000.125):
            row_ptr, col = vpd.build_neighbor_list(cuda(shift + ijk * h), 3 * h)
            row_ptr, col = host(row_ptr), host(col)
            for p in range(n ** 3):
                expected = np.nonzero((d2[p] > 0) & (d2[p] <= 9))[0]
                assert np.array_equal(col[row_ptr[p]:row_ptr[p + 1]], expected)


def test_neighbor_list_matches_reference_fixture():
    ref = np.load(golden("ref_neighbors_jittered.npz"))
    row_ptr, col = vpd.build_neighbor_list(cuda(ref["positions"]), float(ref["horizon"]))
    assert np.array_equal(host(row_ptr), ref["row_ptr"])
    assert np.array_equal(host(col), ref["col"])


def test_neighbor_lists_full_size():
    """The 1M-point jittered bar: the device lists equal the oracle's element for element,
    and are sorted and symmetric."""
    case = tensile_bar(3, precision=0)
    with vpd.Simulation(case) as sim:
        row_ptr, col = sim.neighbors()
        pos = sim.field("position")
    assert 230 < len(col) / len(pos) < 245
    ro, co = O.neighbor_list(pos, case.horizon)
    assert np.array_equal(row_ptr, ro) and np.array_equal(col, co)
    rows = np.repeat(np.arange(len(pos)), np.diff(row_ptr))
    assert np.all(np.diff(col.astype(np.int64) + rows * len(pos)) > 0)  # ascending per row
    fwd = rows.astype(np.int64) * len(pos) + col
    bwd = col.astype(np.int64) * len(pos) + rows
    assert np.array_equal(np.sort(fwd), np.sort(bwd))


# ---------------------------------------------------------------- module functions
@pytest.fixture(scope="module")
def small_block():
    case = tensile_bar(1, nx=12, ny=7, nz=6, jitter=0.05, jitter_seed=5)
    sim = O.OracleSim(case)
    pos, vol = sim.get("position"), sim.get("volume")[:, 0]
    row_ptr, col = sim.neighbors()
    rng = np.random.default_rng(3)
    disp = 0.002 * rng.standard_normal(pos.shape) + 0.003 * pos[:, [0]] * np.array([1.0, -0.3, 0.2])
    return dict(case=case, pos=pos, vol=vol, row_ptr=row_ptr, col=col, disp=disp, rng=rng)


def test_shape_tensor_and_deformation_match_oracle(small_block):
    b = small_block
    rc, kinv_o = O.shape_inverse(b["pos"], b["vol"], b["row_ptr"], b["col"])
    args = [cuda(b["pos"]), cuda(b["vol"]), cuda(b["row_ptr"], torch.int64), cuda(b["col"], torch.int32)]
    kinv = vpd.shape_tensor_inverse(*args)
    assert max_rel(host(kinv), kinv_o) < 1e-13
    F_o = O.deformation(b["pos"], b["disp"], b["vol"], b["row_ptr"], b["col"], kinv_o)
    F = vpd.deformation_gradients(args[0], cuda(b["disp"]), args[1], args[2], args[3], kinv)
    assert np.max(np.abs(host(F) - F_o)) < 1e-12


def test_force_density_matches_oracle(small_block):
    b = small_block
    rng = b["rng"]
    n = len(b["vol"])
    rc, kinv = O.shape_inverse(b["pos"], b["vol"], b["row_ptr"], b["col"])
    F = O.deformation(b["pos"], b["disp"], b["vol"], b["row_ptr"], b["col"], kinv)
    s = rng.standard_normal((n, 3, 3)) * 100.0
    sigma = (s + s.transpose(0, 2, 1)).reshape(n, 9)
    bond = (rng.random(len(b["col"])) < 0.1).astype(np.float64)
    rc, f_o = O.force(b["pos"], b["vol"], b["row_ptr"], b["col"], kinv, F, sigma, bond)
    f = vpd.force_density(cuda(b["pos"]), cuda(b["vol"]), cuda(b["row_ptr"], torch.int64),
                          cuda(b["col"], torch.int32), cuda(kinv), cuda(F), cuda(sigma), cuda(bond))
    assert max_rel(host(f), f_o) < 1e-12


def test_damage_matches_oracle(small_block):
    b = small_block
    disp = b["disp"] * 8.0
    rc, bd_o, idx_o = O.damage(b["pos"], disp, b["vol"], b["row_ptr"], b["col"], 0.01, 0.005,
                               np.zeros(len(b["col"])))
    assert 0 < bd_o.sum() < len(bd_o)
    bd = cuda(np.zeros(len(b["col"])))
    idx = vpd.damage_update(cuda(b["pos"]), cuda(disp), cuda(b["vol"]), cuda(b["row_ptr"], torch.int64),
                            cuda(b["col"], torch.int32), 0.01, 0.005, bd)
    assert np.array_equal(host(bd), bd_o)
    assert np.max(np.abs(host(idx) - idx_o)) < 1e-14


def test_corotational_and_material_match_oracle():
    rng = np.random.default_rng(8)
    n = 777
    I = np.tile(np.eye(3).reshape(1, 9), (n, 1))
    fN = I + 0.01 * rng.standard_normal((n, 9))
    fNP1 = fN + 2e-4 * rng.standard_normal((n, 9))
    vN = I + 0.004 * rng.standard_normal((n, 9))
    th = rng.random(n)
    rN = np.stack([np.cos(th), -np.sin(th), 0 * th, np.sin(th), np.cos(th), 0 * th, 0 * th, 0 * th, 1 + 0 * th], 1)
    dt = 1e-5
    rc, out_o = O.corotational(fN, fNP1, vN, rN, dt)
    out = vpd.corotational_update(cuda(fN), cuda(fNP1), cuda(vN), cuda(rN), dt)
    for k, v in out_o.items():
        assert np.max(np.abs(host(out[k]) - v)) < 1e-9 * max(1.0, np.max(np.abs(v))), k
    # three material increments from rest, the last ones plastic
    props = np.array(REFERENCE_JC_PROPS)
    state_o = dict(defgrad_old=I.copy(), left_stretch=I.copy(), rotation=I.copy(),
                   strain=np.zeros((n, 9)), stress_corotational=np.zeros((n, 9)),
                   state=np.zeros((n, 6)), temperature=np.full(n, 293.0),
                   energy_internal=np.zeros(n), energy_inelastic=np.zeros(n))
    state_g = {k: cuda(v) for k, v in state_o.items()}
    F = I.copy()
    for it in range(3):
        F = F + (0.004 if it else 0.0005) * np.array([1, 0.2, 0, 0.2, -0.3, 0, 0, 0, -0.3]) \
            + 1e-4 * rng.standard_normal((n, 9))
        rc, state_o = O.material_update(props, dt, F, state_o)
        assert rc == 0
        spatial = vpd.material_update(props, dt, cuda(F), state_g)
        for k, v in state_o.items():
            got = host(spatial) if k == "stress_spatial" else host(state_g[k])
            assert max_rel(got, v) < 1e-11, (it, k)
    assert np.max(state_o["state"][:, 1]) > 0.0  # the return map ran


# ---------------------------------------------------------------- full increment
def test_increment_reproduces_archived_pd_coarse():
    """All 4800 increments of the reference's archived JC case."""
    header, g = load_golden_timeseries()
    with vpd.Simulation(pd_coarse()) as sim:
        rows = sim.step(4800)
        snap = np.load(golden("pd_coarse_snapshot.npz"))
        assert max_rel(sim.field("displacement"), snap["displacement"]) < 1e-9
        assert max_rel(sim.field("stress_spatial")[:, 0], snap["axial_stress"]) < 1e-8
        assert max_rel(sim.field("state")[:, 1], snap["eqps"]) < 1e-8
    mine = rows[g[:, 0].astype(int) - 1]
    j = header.index("average_axial_stress_MPa")
    assert nrmse(mine[:, j], g[:, j]) < 1e-6
    for name in ("reaction_force_N", "max_eqps", "kinetic_energy_Nmm", "internal_energy_Nmm",
                 "external_work_Nmm", "lateral_strain", "average_axial_strain"):
        k = header.index(name)
        assert max_rel(mine[:, k], g[:, k]) < 1e-8, name
    assert np.all(mine[:, header.index("finite")] == 1.0)


def test_case_file_runner_reproduces_archived_pd_coarse(tmp_path):
    """The reference's own case file pd_coarse.json run through vpd.runner: the three output
    files come out in the reference's layout, the timeseries has the archived rows and stress
    history, the snapshot has the archived points (reference coordinates to the last printed
    digit) and fields, and the case's acceptance verdict is the archived 'pass'."""
    import csv
    import gzip
    import json
    from vpd.runner import run_boundary_case
    rc = run_boundary_case(golden("cases/pd_coarse.json"), str(tmp_path), golden(""), log=lambda line: None)
    assert rc == 0
    header, g = load_golden_timeseries()
    with open(tmp_path / "timeseries.csv") as f:
        mine = list(csv.reader(f))
    assert mine[0] == ["material"] + header
    vals = np.array([[float(x) for x in r[1:]] for r in mine[1:]])
    assert vals.shape == g.shape and np.array_equal(vals[:, 0], g[:, 0])
    j = header.index("average_axial_stress_MPa")
    assert nrmse(vals[:, j], g[:, j]) < 1e-6
    with open(tmp_path / "field_snapshots.csv") as f:
        snap = list(csv.reader(f))
    with gzip.open(golden("pd_coarse_snapshot_head.csv.gz"), "rt") as f:
        head = list(csv.reader(f))
    assert snap[0] == head[0] and len(snap) == 1 + 1683
    for a, b in zip(snap[1:], head[1:]):
        assert a[:7] == b[:7]  # material, step, time, particle, x0 y0 z0
    col = {k: i for i, k in enumerate(head[0])}
    ref = np.load(golden("pd_coarse_snapshot.npz"))

    def arr(*names):
        return np.array([[float(r[col[k]]) for k in names] for r in snap[1:]])

    assert max_rel(arr("ux_mm", "uy_mm", "uz_mm"), ref["displacement"]) < 1e-9
    assert max_rel(arr("vx_mm_per_ms", "vy_mm_per_ms", "vz_mm_per_ms"), ref["velocity"]) < 1e-6
    assert max_rel(arr("axial_stress_MPa")[:, 0], ref["axial_stress"]) < 1e-8
    assert max_rel(arr("axial_strain")[:, 0], ref["axial_strain"]) < 1e-8
    assert max_rel(arr("eqps")[:, 0], ref["eqps"]) < 1e-8
    with open(tmp_path / "metadata.json") as f:
        meta = json.load(f)
    assert meta["status"] == "pass" and meta["particles"] == 1683
    assert meta["materials"][0]["maxEqps"] == pytest.approx(0.0278018224371612, rel=1e-8)
    assert meta["materials"][0]["finalReaction_N"] == pytest.approx(9875.54163611348, rel=1e-8)


def test_increment_matches_reference_library_jittered_damage():
    ref = np.load(golden("ref_tensile_bar_1.npz"))
    bar = tensile_bar(1, jitter=0.05, jitter_seed=7, damage_mode=1, damage_initiation=0.004)
    with vpd.Simulation(bar) as sim:
        rows = sim.step(300)
        assert nrmse(rows[:, STRESS], ref["diag"][:, STRESS]) < 1e-6
        assert max_rel(sim.field("displacement"), ref["displacement"]) < 1e-9
        assert max_rel(sim.field("stress_corotational"), ref["stress_corotational"]) < 1e-8
        assert np.array_equal(sim.field("damage_index"), ref["damage_index"])
        state = sim.field("state")
    assert np.mean(state[:, 5] == ref["state"][:, 5]) > 0.999  # JC iteration counts


def test_increment_matches_oracle_full_tensile_bar_1():
    """The 40x10x10 bar over its full 2000 increments (plastic)."""
    case = tensile_bar(1)
    with vpd.Simulation(case) as sim:
        rows = sim.step(case.steps)
        fields = {f: sim.field(f) for f in ("displacement", "stress_spatial", "state")}
    o = O.OracleSim(case)
    ref = o.step(case.steps)
    assert ref[-1, vpd.DIAG["max_eqps"]] > 1e-3
    assert nrmse(rows[:, STRESS], ref[:, STRESS]) < 1e-6
    assert nrmse(fields["displacement"], o.get("displacement")) < 1e-6
    assert nrmse(fields["state"][:, 1], o.get("state")[:, 1]) < 1e-6
    assert nrmse(fields["stress_spatial"], o.get("stress_spatial")) < 1e-6


def test_sliced_ell_layout_matches_stencil_layout(monkeypatch):
    """The sliced-ELL bond layout (used when points do not form the lattice in index order)
    gives the same increments as the lattice-stencil layout."""
    case = tensile_bar(1, jitter=0.05, jitter_seed=7, damage_mode=1, damage_initiation=0.004)
    with vpd.Simulation(case) as a:
        ra = a.step(200)
        ua, da = a.field("displacement"), a.field("damage_index")
    monkeypatch.setenv("VPD_BOND_LAYOUT", "ell")
    with vpd.Simulation(case) as b:
        rb = b.step(200)
        assert nrmse(rb[:, STRESS], ra[:, STRESS]) < 1e-9
        assert max_rel(b.field("displacement"), ua) < 1e-9
        assert np.array_equal(b.field("damage_index"), da)


def test_horizon_beyond_the_stencil_windows_uses_the_generic_layout():
    """A horizon of 15 spacings on a 32-point-wide lattice makes stencil groups of 31 slots, more
    than the tiled kernels' 32-bit windows hold for several points per thread: the case runs on
    the sliced-ELL layout instead, and matches the oracle."""
    case = tensile_bar(1, nx=8, ny=32, nz=4, horizon=15.015 * 0.5)
    with vpd.Simulation(case) as sim:
        assert sim.layout_words == 0
        rows = sim.step(20)
        u = sim.field("displacement")
    o = O.OracleSim(case)
    ref = o.step(20)
    assert nrmse(rows[:, STRESS], ref[:, STRESS]) < 1e-9
    assert max_rel(u, o.get("displacement")) < 1e-9


@pytest.mark.parametrize("dims", [(24, 21, 17), (12, 37, 70)])
@pytest.mark.parametrize("kind", ["", "staged", "staged4", "tiled2"])
@pytest.mark.parametrize("damage", [0, 1])
def test_tiled_fp64_bond_kernels_match_slot_kernels_bitwise(monkeypatch, damage, kind, dims):
    """The tiled FP64 bond kernels (two points per thread along y; in the force kernel four
    through L1 by default, two with tiled2, or two or four from a shared-memory box filled plane
    by plane by TMA with staged) sum every point's bonds in the per-slot kernels' order with
    the same operations:
    on the jittered horizon-4 bar (y extent 21 and z extent 17, so the last tiles are ragged)
    the increments agree bit for bit, bond breaking included. The second lattice (z extent 70)
    takes three staged tiles along z and three along y, the last of each ragged."""
    nx, ny, nz = dims
    case = tensile_bar(3, nx=nx, ny=ny, nz=nz, damage_mode=damage, damage_initiation=0.004,
                       precision=PRECISION_FP64)
    fields = ("displacement", "velocity", "stress_corotational", "state", "damage_index")
    monkeypatch.setenv("VPD_BOND_KERNEL", "slot")
    with vpd.Simulation(case) as a:
        ra = a.step(150)
        fa = {f: a.field(f) for f in fields}
    monkeypatch.setenv("VPD_BOND_KERNEL", "staged" if kind.startswith("staged") else kind)
    if kind == "staged4":
        monkeypatch.setenv("VPD_STAGED", "4x128")
    with vpd.Simulation(case) as b:
        rb = b.step(150)
        for f in fields:
            assert np.array_equal(b.field(f), fa[f]), f
    assert np.array_equal(ra, rb)
    if damage:
        assert fa["damage_index"].max() > 0


def test_graph_and_stage_launches_agree_bitwise():
    case = tensile_bar(1, jitter=0.05, jitter_seed=9, damage_mode=1, damage_initiation=0.003)
    with vpd.Simulation(case) as a, vpd.Simulation(case) as b:
        ra = a.step(40)
        b.profile_stages(40)
        for f in ("displacement", "velocity", "stress_corotational", "state", "damage_index"):
            assert np.array_equal(a.field(f), b.field(f)), f
        with vpd.Simulation(case) as c:
            assert np.array_equal(c.step(40), ra)  # run to run determinism


# ---------------------------------------------------------------- plugin ABI
def test_vumat_plugin_matches_restated_plugin():
    """vumat_adapter_call of libvpd_gpu.so vs the restated Fortran plugin on plastic blocks of
    1, 255, 256, 257 and 513 rows, two increments each."""
    gpu, cpu = vpd.library(), O.oracle_lib()
    rng = np.random.default_rng(4)
    props = np.array(REFERENCE_JC_PROPS)
    for nb in (1, 255, 256, 257, 513):
        stress = 300 * rng.standard_normal((nb, 6))
        state = np.column_stack([np.ones(nb), 0.01 * rng.random(nb), 293 + 50 * rng.random(nb),
                                 300 + 50 * rng.random(nb), 1e-5 * rng.random(nb), np.zeros(nb)])
        args = (props, 2.5e-5, 2e-3 * rng.standard_normal((nb, 6)), stress, state,
                np.full(nb, 300.0), rng.random(nb), rng.random(nb))
        a, b = O.vumat_block(gpu, *args), O.vumat_block(cpu, *args)
        for k in a:
            assert max_rel(a[k], b[k]) < 1e-10, (nb, k)
        assert np.mean(a["state"][:, 5] == b["state"][:, 5]) > 0.99


def test_vumat_plugin_thermal_units():
    ref = np.load(golden("ref_jc_thermal.npz"))
    for tag, w2h in (("legacy", 1.0), ("scaled", 1.0e6)):
        props = np.array(REFERENCE_JC_PROPS[:13] + (w2h,))
        first = O.vumat_block(vpd.library(), props, 2.5e-5, np.zeros((1, 6)), np.zeros((1, 6)),
                              np.zeros((1, 6)), np.array([293.0]), np.zeros(1), np.zeros(1))
        inc = np.zeros((1, 6))
        inc[0, 0] = 400 * 2.5e-5
        out = O.vumat_block(vpd.library(), props, 2.5e-5, inc, first["stress"], first["state"],
                            first["temperature"], first["energy_internal"], first["energy_inelastic"])
        for k, v in out.items():
            assert max_rel(v, ref[f"{tag}_{k}"]) < 1e-12, (tag, k)


@pytest.mark.skipif(not O.reference_available(), reason="reference library not built")
def test_reference_adapter_runs_on_the_gpu_plugin():
    """The reference's own VumatPdCorrespondenceMaterial, dlopening libvpd_gpu.so as its plugin,
    reproduces its run with the restated CPU plugin."""
    case = pd_coarse().replace(steps=300)
    a = O.RefSim(case, plugin=vpd.library_path())
    b = O.RefSim(case)
    ra, rb = a.step(300), b.step(300)
    assert nrmse(ra[:, STRESS], rb[:, STRESS]) < 1e-9
    assert max_rel(a.get("state"), b.get("state")) < 1e-9


# ---------------------------------------------------------------- errors, host-injected
def test_singular_shape_tensor_reported():
    case = tensile_bar(1, horizon=0.4)  # horizon below the spacing: no bonds, K = 0
    with pytest.raises(vpd.VpdError) as e:
        vpd.Simulation(case)
    assert e.value.status == 3


def test_nonfinite_positions_reported():
    case = tensile_bar(1)
    pos = O.OracleSim(case).get("position")
    pos[17, 1] = np.nan
    with pytest.raises(vpd.VpdError) as e:
        vpd.Simulation(case, positions=pos)
    assert e.value.status == 4


def test_affine_completeness_on_device():
    case = Case(name="cube", nx=9, ny=9, nz=9, spacing=1.0, horizon=2.0, dt=1e-5, steps=1,
                density=1.0, props=REFERENCE_JC_PROPS, grip_velocity=1.0, ramp_time=1.0)
    sim = O.OracleSim(case)
    x, vol = sim.get("position"), sim.get("volume")[:, 0]
    row_ptr, col = sim.neighbors()
    args = [cuda(x), cuda(vol), cuda(row_ptr, torch.int64), cuda(col, torch.int32)]
    kinv = vpd.shape_tensor_inverse(*args)
    u = np.stack([0.02 * x[:, 0] + 0.03 * x[:, 1], -0.01 * x[:, 1], 0.04 * x[:, 2]], 1)
    F = host(vpd.deformation_gradients(args[0], cuda(u), args[1], args[2], args[3], kinv))
    assert np.max(np.abs(F - np.array([1.02, 0.03, 0, 0, 0.99, 0, 0, 0, 1.04]))) < 1e-12
