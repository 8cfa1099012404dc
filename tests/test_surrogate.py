"""The learned Johnson-Cook return map, through the C ABI.

* The training increments are the device VUMAT's own results: a sample of them is re-solved
  by the CPU restatement of the VUMAT (oracle/jc_vumat.c) and must agree.
* Training (vpd_train_surrogate: the tcgen05 forward/backward kernels and Adam on the GPU, on
  2M increments, batch 8192, 20 epochs, lr 1e-3) must converge, and the trained network on
  the device must equal the CPU FP64 network (oracle/mlp.py) on the same weights.
* In the loop (the 4000-point bar, 2000 increments into plastic flow), every accepted
  increment meets the VUMAT's own residual tolerance, so the stress history stays within
  1e-6 of the plain run (bound 5e-3).
* What the network gains over the method without it: against the VUMAT's bisection, the
  network guess with two Newton steps cuts the yield-function evaluations by more than 3x;
  against a warm start from the previous plastic increment alone, the hybrid guess (network
  where a point has no plastic history) sends fewer increments to the bisection fallback.
"""
import numpy as np
import pytest

from conftest import nrmse

import mlp as M
import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def vpd_mod():
    import vpd
    return vpd


def props():
    from vpd.case import tensile_bar
    return np.array(tensile_bar(1).props)


@pytest.fixture(scope="module")
def trained():
    vpd = vpd_mod()
    w, b, rep = vpd.train_surrogate(props(), samples=2_000_000, epochs=20, batch=8192,
                                    learning_rate=1e-3, seed=2026, validation_fraction=0.05)
    return w, b, rep


def test_samples_are_vumat_increments():
    vpd = vpd_mod()
    p = props()
    f, t, r = vpd.surrogate_samples(p, 7, 2048, records=True)
    assert np.isfinite(f).all() and np.isfinite(t).all() and np.isfinite(r).all()
    assert (f[:, 10:] == 0).all() and (t[:, 7:15] == 0).all()
    plastic = t[:, 15] == 1.0
    assert 0.3 < plastic.mean() < 0.8
    assert np.array_equal(plastic, r[:, 24] == 1.0)
    assert (t[plastic, 0] > 0).all() and (t[plastic, 0] < 1.2).all()  # epInc / xf
    lib = O.oracle_lib()
    for k in range(0, 2048, 8):
        state = np.array([[1.0, r[k, 12], r[k, 13], r[k, 14], 0.0, 0.0]])
        out = O.vumat_block(lib, p, r[k, 15], r[k, 0:6][None], r[k, 6:12][None], state,
                            np.array([r[k, 13]]), np.zeros(1), np.zeros(1))
        assert np.max(np.abs(out["stress"][0] - r[k, 16:22])) < 1e-9 * max(1.0, r[k, 14])
        assert abs(out["state"][0, 4] - r[k, 22]) <= 1e-15 + 1e-12 * abs(r[k, 22])
        assert out["state"][0, 5] == r[k, 23]  # same bisection iteration count


def test_training_converges(trained):
    _, _, rep = trained
    loss = rep["epoch_loss"]
    assert len(loss) == 20 and np.isfinite(loss).all()
    assert loss[-1] < loss[0] / 3
    assert rep["validation_loss"] < 1.5 * loss[-1]
    assert rep["ratio_rmse"] < 0.05
    assert 0.3 < rep["plastic_fraction"] < 0.8


def test_trained_network_on_device_equals_cpu_network(trained):
    vpd = vpd_mod()
    w, b, _ = trained
    f, t, _ = vpd.surrogate_samples(props(), 99, 4096)
    dev = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a)).to("cuda", dt)
    out = vpd.mlp_forward(dev(w.view(np.int16), torch.int16), dev(b, torch.float32),
                          dev(f, torch.float32)).cpu().numpy()
    ref = M.forward(w, b, f)
    assert np.linalg.norm(out - ref) < 2e-3 * np.linalg.norm(ref)
    plastic = t[:, 15] == 1.0
    assert np.sqrt(np.mean((out[plastic, 0] - t[plastic, 0]) ** 2)) < 0.05  # held-out seed


def run_bar(steps, mode=None, weights=None):
    vpd = vpd_mod()
    from vpd.case import MATERIAL_SURROGATE, tensile_bar
    case = tensile_bar(1, material_mode=MATERIAL_SURROGATE if mode else 0)
    with vpd.Simulation(case) as sim:
        if mode:
            w, b = weights if mode[0] != "warm_start" else (None, None)
            sim.set_surrogate(w, b, guess=mode[0], newton_steps=mode[1])
        rows = sim.step(steps)
        state = sim.field("state")
    return rows, state


@pytest.fixture(scope="module")
def bar_runs(trained):
    w, b, _ = trained
    runs = {"vumat": run_bar(2000)}
    for mode in (("network", 2), ("hybrid", 2), ("warm_start", 2)):
        runs[mode[0]] = run_bar(2000, mode, (w, b))
    return runs


def test_surrogate_in_loop_matches_vumat(bar_runs):
    vpd = vpd_mod()
    ref_rows, ref_state = bar_runs["vumat"]
    col = vpd.DIAG["average_axial_stress_MPa"]
    assert ref_state[:, 1].max() > 1e-3  # the bar flows plastically
    for name in ("network", "hybrid", "warm_start"):
        rows, state = bar_runs[name]
        assert rows[-1, vpd.DIAG["finite"]] == 1.0
        assert nrmse(rows[:, col], ref_rows[:, col]) < 5e-3      # the tolerance stated for the surrogate
        assert nrmse(rows[:, col], ref_rows[:, col]) < 1e-6      # what the residual gate delivers
        # each accepted increment lies within the VUMAT's tolerance band (|r| < E 1e-9), as the
        # bisection's does, at a different point of it: eqps agrees to ~1e-6 relative
        assert np.max(np.abs(state[:, 1] - ref_state[:, 1])) < 1e-4 * ref_state[:, 1].max()
        plastic = rows[:, vpd.DIAG["plastic_points"]].sum()
        ref_plastic = ref_rows[:, vpd.DIAG["plastic_points"]].sum()
        assert abs(plastic - ref_plastic) <= 1e-4 * ref_plastic
    assert ref_rows[:, vpd.DIAG["fallback_points"]].sum() == 0


def test_what_the_network_gains(bar_runs):
    vpd = vpd_mod()
    evals = {k: v[1][:, 5].sum() for k, v in bar_runs.items()}  # VUMAT state 6: iterations
    fallback = {k: v[0][:, vpd.DIAG["fallback_points"]].sum() for k, v in bar_runs.items()}
    plastic = bar_runs["vumat"][0][:, vpd.DIAG["plastic_points"]].sum()
    print("yield evaluations", evals, "fallback points", fallback, "plastic points", plastic)
    # over the VUMAT's bisection (no network): the network's guess converges in two Newton steps
    # for most points and cuts the yield-function evaluations by more than 3x
    assert fallback["network"] < 0.1 * plastic
    assert evals["network"] < evals["vumat"] / 3
    # over the warm start alone: the network covers the points without plastic history
    assert fallback["hybrid"] < fallback["warm_start"]
    assert evals["hybrid"] <= evals["warm_start"]


def test_surrogate_api_errors(trained):
    vpd = vpd_mod()
    from vpd.case import MATERIAL_SURROGATE, tensile_bar
    w, b, _ = trained
    with vpd.Simulation(tensile_bar(1)) as sim:
        with pytest.raises(vpd.VpdError):
            sim.set_surrogate(w, b)  # not a surrogate case
    with vpd.Simulation(tensile_bar(1, material_mode=MATERIAL_SURROGATE)) as sim:
        with pytest.raises(vpd.VpdError):
            sim.step(1)  # no surrogate attached
        with pytest.raises(vpd.VpdError):
            sim.set_surrogate(None, None, guess="network")
        with pytest.raises(vpd.VpdError):
            sim.set_surrogate(w, b, newton_steps=-1)
        sim.set_surrogate(None, None, guess="warm_start")
        assert sim.step(3).shape == (3, len(vpd.DIAG_COLUMNS))
    with pytest.raises(vpd.VpdError):
        vpd.train_surrogate(props(), samples=1000, batch=8192)
