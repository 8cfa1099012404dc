import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "vumat-pd_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libvpd_gpu.so")
    config.addinivalue_line("markers", "late: runs after the other tests, so that a failure under -x "
                                       "leaves their results in place (tests not yet run on a GPU)")


def pytest_collection_modifyitems(session, config, items):
    # stable: `late` tests after the others, and the no-allocation entry point's file last of all
    items.sort(key=lambda item: (os.path.basename(str(item.fspath)) == "test_zz_no_alloc.py",
                                 item.get_closest_marker("late") is not None))


def golden(name):
    return os.path.join(GOLDEN, name)


def nrmse(a, ref):
    """RMS difference over peak |reference| (analyse_and_plot.py:66-74)."""
    a, ref = np.asarray(a, float), np.asarray(ref, float)
    peak = np.max(np.abs(ref))
    return float(np.sqrt(np.mean((a - ref) ** 2)) / (peak if peak > 0 else 1.0))


def max_rel(a, ref):
    a, ref = np.asarray(a, float), np.asarray(ref, float)
    scale = np.max(np.abs(ref))
    return float(np.max(np.abs(a - ref)) / (scale if scale > 0 else 1.0))


def load_golden_timeseries():
    import csv
    import gzip
    with gzip.open(golden("pd_coarse_timeseries.csv.gz"), "rt") as f:
        rows = list(csv.reader(f))
    return rows[0][1:], np.array([[float(x) for x in r[1:]] for r in rows[1:]])


def build_abi_host(out_dir):
    """Compiles tests/abi_host.cpp (the C++ host on include/vpd_gpu.h) against the in-tree
    libvpd_gpu.so with the system compiler; returns the executable's path."""
    import subprocess
    lib_dir = os.path.join(ROOT, "vumat-pd_b200")
    exe = os.path.join(str(out_dir), "abi_host")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "abi_host.cpp"), "-o", exe,
                    os.path.join(lib_dir, "libvpd_gpu.so"), f"-Wl,-rpath,{lib_dir}"], check=True)
    return exe


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    return O
