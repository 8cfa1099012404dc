"""The C ABI driven by a compiled C++ host (tests/abi_host.cpp: include/vpd_gpu.h only, linked
to libvpd_gpu.so), as the reference's host would drive it in place of runMaterial's loop: its
50 increments of the 40x10x10 steel bar, stepped in chunks of 10, equal the Python binding's
run of the same case bit for bit, rows and final displacement."""
import subprocess

import numpy as np
import pytest

from conftest import build_abi_host

import vpd
from vpd.case import tensile_bar

pytestmark = pytest.mark.gpu


def test_cpp_host_runs_the_increment_through_the_c_abi(tmp_path):
    exe = build_abi_host(tmp_path)
    out = tmp_path / "run.bin"
    text = subprocess.run([exe, "run", "50", str(out)], capture_output=True, text=True,
                          check=True).stdout
    case = tensile_bar(1)
    words = text.split()
    assert int(words[1]) == case.n_points and float(words[3]) == case.dt
    data = np.fromfile(out, dtype=np.float64)
    rows = data[: 50 * len(vpd.DIAG)].reshape(50, len(vpd.DIAG))
    u = data[50 * len(vpd.DIAG):].reshape(-1, 3)
    with vpd.Simulation(case) as sim:
        ref_rows = sim.step(50)
        ref_u = sim.field("displacement")
    assert np.array_equal(rows, ref_rows)
    assert np.array_equal(u, ref_u)
    assert rows[-1, vpd.DIAG["step"]] == 50 and np.abs(u).max() > 0
