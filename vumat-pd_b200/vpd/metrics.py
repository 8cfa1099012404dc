"""The PD half of the reference's tensile benchmark analysis, restated.

The reference recomputes its validation metrics from the runner's output files with
benchmarks/tensile3d/analyse_and_plot.py and checks them against its frozen values with
verify_metrics.py (0.5 % relative, absolute 1e-8). The FEM solver whose run is the reference
solution is out of scope here, so this module computes only the PD cases' metrics, against an
FEM reference given as data (its archived outputs, or the arrays derived from them):

  stress_MPa          last window-mean axial stress of the run
  mean_axial_strain   last window-mean axial strain
  max_eqps            last max equivalent plastic strain
  stress_history_pct  RMS over the 240 common output times (0.0005 ms apart) of the axial
                      stress difference to the FEM reference, over its peak |stress|, in %
  displacement_pct    RMS over the 1551 sample coordinates of the displacement difference
                      (trilinear interpolation of the nodal grid), over 2 mm, in %
  max_eqps_pct        |max eqps - the FEM reference's| over the FEM reference's, in %
  final_stress_pct    |last stress - the FEM reference's last stress| over the latter, in %
  nodes               number of snapshot rows

(analyse_and_plot.py:44-82; verify_metrics.py:9-13.) No plots: matplotlib is not needed.

    python -m vpd.metrics RESULTS_DIR FEM_REFERENCE_DIR
"""
from __future__ import annotations

import csv
import json
import os
import sys

import numpy as np

COMMON_TIMES = np.arange(1, 241) * 0.0005
REL_TOL, ABS_TOL = 0.005, 1e-8  # verify_metrics.py:11-12


def sample_coordinates() -> np.ndarray:
    """x = 4, 6, ..., 96 mm; y = -10, ..., 10 mm; z = -2, 0, 2 mm, x slowest (1551 rows)."""
    x, y, z = np.arange(4.0, 98.0, 2.0), np.arange(-10.0, 12.0, 2.0), np.array([-2.0, 0.0, 2.0])
    grid = np.stack(np.meshgrid(x, y, z, indexing="ij"), -1).reshape(-1, 3)
    assert len(grid) == 1551
    return grid


def read_csv(path: str) -> dict:
    """Numeric columns of a CSV file (plain or gzipped) as float arrays."""
    import gzip
    opener = gzip.open if path.endswith(".gz") else open
    with opener(path, "rt") as f:
        rows = list(csv.reader(f))
    out = {}
    for j, name in enumerate(rows[0]):
        try:
            out[name] = np.array([float(r[j]) for r in rows[1:]])
        except ValueError:
            pass
    return out


def interpolate_nodes(nodes: dict, query: np.ndarray) -> np.ndarray:
    """Displacement (ux, uy, uz) at the query points by trilinear interpolation on the nodal
    grid spanned by the distinct reference coordinates x0_mm, y0_mm, z0_mm of ``nodes``."""
    ref = np.stack([nodes["x0_mm"], nodes["y0_mm"], nodes["z0_mm"]], 1)
    axes = [np.unique(ref[:, d]) for d in range(3)]
    shape = tuple(len(a) for a in axes)
    cell = np.stack([np.searchsorted(axes[d], ref[:, d]) for d in range(3)], 1)
    u = np.zeros(shape + (3,))
    u[cell[:, 0], cell[:, 1], cell[:, 2]] = np.stack([nodes["ux_mm"], nodes["uy_mm"], nodes["uz_mm"]], 1)
    lo, frac = [], []
    for d in range(3):
        j = np.clip(np.searchsorted(axes[d], query[:, d], side="right") - 1, 0, len(axes[d]) - 2)
        t = (query[:, d] - axes[d][j]) / (axes[d][j + 1] - axes[d][j])
        if t.min() < -1e-8 or t.max() > 1 + 1e-8:
            raise ValueError("sample coordinates outside the nodal grid")
        lo.append(j)
        frac.append(t)
    out = np.zeros((len(query), 3))
    for corner in range(8):
        bits = [(corner >> d) & 1 for d in range(3)]
        w = np.ones(len(query))
        for d in range(3):
            w *= frac[d] if bits[d] else 1.0 - frac[d]
        out += w[:, None] * u[lo[0] + bits[0], lo[1] + bits[1], lo[2] + bits[2]]
    return out


def fem_reference(fem_dir: str) -> dict:
    """What the metrics read of the FEM reference's archived outputs (timeseries.csv and
    final_nodes.csv, plain or gzipped)."""
    def find(name):
        for cand in (name, name + ".gz"):
            if os.path.exists(os.path.join(fem_dir, cand)):
                return os.path.join(fem_dir, cand)
        raise FileNotFoundError(os.path.join(fem_dir, name))
    ts = read_csv(find("timeseries.csv"))
    nodes = read_csv(find("final_nodes.csv"))
    return {"stress": np.interp(COMMON_TIMES, ts["time_ms"], ts["average_axial_stress_MPa"]),
            "final_stress": float(ts["average_axial_stress_MPa"][-1]),
            "max_eqps": float(ts["max_eqps"][-1]),
            "u": interpolate_nodes(nodes, sample_coordinates())}


def pd_metrics(series: dict, u_samples: np.ndarray, n_nodes: int, ref: dict) -> dict:
    """The metrics of one PD run: ``series`` its timeseries columns, ``u_samples`` its final
    displacement at sample_coordinates(), ``ref`` the FEM reference (fem_reference())."""
    stress = np.interp(COMMON_TIMES, series["time_ms"], series["average_axial_stress_MPa"])
    peak = float(np.max(np.abs(ref["stress"])))
    last_stress = float(series["average_axial_stress_MPa"][-1])
    max_eqps = float(series["max_eqps"][-1])
    return {
        "stress_MPa": last_stress,
        "mean_axial_strain": float(series["average_axial_strain"][-1]),
        "max_eqps": max_eqps,
        "stress_history_pct": float(100.0 * np.sqrt(np.mean((stress - ref["stress"]) ** 2)) / peak),
        "displacement_pct": float(100.0 * np.sqrt(np.mean(np.sum((u_samples - ref["u"]) ** 2, 1))) / 2.0),
        "max_eqps_pct": float(100.0 * abs(max_eqps - ref["max_eqps"]) / ref["max_eqps"]),
        "final_stress_pct": float(100.0 * abs(last_stress - ref["final_stress"]) / abs(ref["final_stress"])),
        "nodes": int(n_nodes),
    }


def run_metrics(results_dir: str, ref: dict) -> dict:
    """pd_metrics of a runner output directory (timeseries.csv, field_snapshots.csv)."""
    series = read_csv(os.path.join(results_dir, "timeseries.csv"))
    snap = read_csv(os.path.join(results_dir, "field_snapshots.csv"))
    last = snap["step"] == snap["step"].max()
    nodes = {k: v[last] for k, v in snap.items()}
    return pd_metrics(series, interpolate_nodes(nodes, sample_coordinates()), int(last.sum()), ref)


def mismatches(expected: dict, actual: dict) -> list:
    """The metric names whose values differ beyond verify_metrics.py's tolerance."""
    import math
    return [k for k, v in expected.items()
            if not math.isclose(v, actual[k], rel_tol=REL_TOL, abs_tol=ABS_TOL)]


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 2:
        print(__doc__.strip().splitlines()[-1].strip(), file=sys.stderr)
        return 1
    print(json.dumps(run_metrics(argv[0], fem_reference(argv[1])), indent=1))
    return 0


if __name__ == "__main__":
    sys.exit(main())
