"""The C-ABI boundary without a GPU: the library loads, exports every entry point the header
declares, the Python struct mirrors the C struct byte for byte, and invalid cases are
rejected on the host before any device work (as the reference's config checks)."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, build_abi_host

import vpd
from vpd.case import VpdCase, pd_coarse, stable_dt, tensile_bar

HEADER = os.path.join(ROOT, "include", "vpd_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(vpd_[a-z_]+|vumat_adapter_call)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_entry_point():
    lib = vpd.library()
    names = declared_functions()
    assert "vpd_create" in names and "vumat_adapter_call" in names and len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert lib.vpd_abi_version() == 1


def c_layout(ctype: str, fields):
    """sizeof and offsetof of a header struct, from a small C program."""
    prog = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void){",
            f'printf("%zu\\n", sizeof({ctype}));']
    prog += [f'printf("%zu\\n", offsetof({ctype}, {f}));' for f in fields]
    prog.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        open(src, "w").write("\n".join(prog))
        subprocess.run(["gcc", src, "-o", exe], check=True)
        return [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]


@pytest.mark.parametrize("ctype,pytype", [("vpd_case", VpdCase),
                                          ("vpd_surrogate_config", vpd.SurrogateConfig),
                                          ("vpd_surrogate_report", vpd.SurrogateReport)])
def test_struct_layouts_match_c(ctype, pytype):
    fields = [f[0] for f in pytype._fields_]
    out = c_layout(ctype, fields)
    assert out[0] == ctypes.sizeof(pytype)
    assert out[1:] == [getattr(pytype, f).offset for f in fields]


def test_compiled_cpp_host_sees_the_python_struct_layout(tmp_path):
    """tests/abi_host.cpp, the C++ host compiled against the header and linked to the library,
    reports the vpd_case layout the ctypes mirror (vpd.case.VpdCase) assumes."""
    exe = build_abi_host(tmp_path)
    out = subprocess.run([exe, "layout"], capture_output=True, text=True, check=True).stdout
    layout = dict((k, int(v)) for k, v in (line.split() for line in out.splitlines()))
    assert layout.pop("sizeof") == ctypes.sizeof(VpdCase)
    assert layout == {f[0]: getattr(VpdCase, f[0]).offset for f in VpdCase._fields_}


def test_invalid_cases_rejected_on_host():
    lib = vpd.library()
    bad = [pd_coarse().replace(nx=1), pd_coarse().replace(horizon=0.0),
           pd_coarse().replace(dt=-1.0), pd_coarse().replace(rise_time=0.0),
           tensile_bar(1, ramp_time=0.0), tensile_bar(1, damage_mode=1, damage_initiation=0.0),
           pd_coarse().replace(nstatev=3), pd_coarse().replace(observation_min=1.0)]
    for case in bad:
        with pytest.raises(vpd.VpdError) as e:
            vpd.Simulation(case)
        assert e.value.status == 1, case
    h = ctypes.c_void_p()
    assert lib.vpd_create(None, None, None, ctypes.byref(h)) == 1
    assert "NULL" in lib.vpd_last_error().decode()


def test_case_builders():
    c1, c2, c3 = tensile_bar(1), tensile_bar(2), tensile_bar(3)
    assert (c1.n_points, c2.n_points, c3.n_points) == (4000, 500000, 1000000)
    assert abs(c1.dt - 6.8302e-5) < 1e-8 and abs(c3.dt - 1.3660e-5) < 1e-8
    assert abs(stable_dt(0.5) / 0.5 - stable_dt(0.1) / 0.1) < 1e-15
    assert c3.props[13] == 1.0e6 and c3.jitter == 0.05 and c3.damage_initiation == 0.02
    assert abs(c3.ramp_time - 200 * c3.dt) < 1e-18


def test_no_silent_fallback_when_library_missing(monkeypatch):
    monkeypatch.setattr(vpd, "_lib", None)
    monkeypatch.setattr(vpd, "library_path", lambda: "/nonexistent/libvpd_gpu.so")
    with pytest.raises(vpd.VpdError):
        vpd.Simulation(tensile_bar(1))
