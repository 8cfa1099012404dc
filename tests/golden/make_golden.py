"""Regenerates the golden fixtures in this directory from the reference checkout.

Run here (where the reference sources are mounted) after `make -C oracle`:

    python tests/golden/make_golden.py REFERENCE_CHECKOUT [--cases-only | --examples]

Fixtures (read by the tests; nothing at test time reads the reference checkout):
  pd_coarse_timeseries.csv.gz  the reference's archived JC run
                               benchmarks/tensile3d/raw/pd_coarse/timeseries.csv.gz (copied)
  pd_coarse_snapshot.npz       the final-step nodal fields of that run
                               (raw/pd_coarse/field_snapshots.csv.gz, step 4800)
  ref_neighbors_jittered.npz   buildNeighborList of the reference library on a jittered
                               17x9x5 lattice (delta = 3.015 h)
  ref_tensile_bar_1.npz        the reference library (via oracle/_ref/libvpd_refharness.so,
                               restated JC plugin) on the 40x10x10 velocity-ramp bar with
                               +-0.05 h jitter and critical-stretch damage: 300 timeseries rows
                               and the final displacement, stress and state
  ref_jc_thermal.npz           one plastic step of the restated JC plugin (pinned bit for bit
                               to the archived run above) with the inputs of the reference's
                               tests/jc_thermal_units_test.cpp, for workToHeat 1 and 1e6
  cases/*.json                 the reference's case files benchmarks/tensile3d/cases/*.json
                               (copied), and configs/johnson_cook.json, the material config they
                               name, under the same relative path
  pd_coarse_snapshot_head.csv.gz  the header and first 200 rows of the archived
                               raw/pd_coarse/field_snapshots.csv.gz (its text, for the writer)

  examples/*.json, configs/elastic.json  the reference's example cases (examples/*.json,
                               copied) and the second material config they name
  example_outputs/<case>/*.gz  the reference's own CLI (oracle/_ref/vumat_pd_run, built from its
                               sources by oracle/Makefile, plugins the restated JC and elastic
                               routines) run on each example case: its output files, gzipped

  ref_config3_slab.npz         the reference library on a 24-plane slab of the jittered 1M-point
                               steel bar (24x50x50 points, horizon 4.015 h, +-0.05 h jitter,
                               workToHeat 1e6, grips at 5 m/s, critical stretch 0.02), FP64:
                               160 timeseries rows, the final damage index of every point, and
                               the final displacement, corotational stress and state (eqps,
                               iteration count) of every 13th point
  archived_pd_cases.npz        for each archived PD case (raw/pd_*): its timeseries, its final
                               displacement interpolated at the analysis script's 1551 sample
                               coordinates (analyse_and_plot.py:46-66), and the archived FEM
                               reference (raw/fem_reference) as those metrics read it: its axial
                               stress at the 240 common output times, its final displacement at
                               the sample coordinates, its last stress and max eqps
  expected_pd_metrics.json     the PD rows of benchmarks/tensile3d/expected/analysis.json

`--cases-only` refreshes only cases/, configs/ and the snapshot head; `--examples` only the
example cases and their outputs; `--config3` only ref_config3_slab.npz; `--archived` only the
archived PD case fixtures.
"""
import csv
import gzip
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "vumat-pd_b200"))


def copy_cases(reference):
    """The case files, their material config and the head of the archived snapshot file."""
    src = os.path.join(reference, "benchmarks", "tensile3d", "cases")
    os.makedirs(os.path.join(HERE, "cases"), exist_ok=True)
    for name in sorted(os.listdir(src)):
        if name.endswith(".json"):
            shutil.copyfile(os.path.join(src, name), os.path.join(HERE, "cases", name))
    os.makedirs(os.path.join(HERE, "configs"), exist_ok=True)
    shutil.copyfile(os.path.join(reference, "configs", "johnson_cook.json"),
                    os.path.join(HERE, "configs", "johnson_cook.json"))
    raw = os.path.join(reference, "benchmarks", "tensile3d", "raw", "pd_coarse")
    with gzip.open(os.path.join(raw, "field_snapshots.csv.gz"), "rt") as f:
        head = [next(f) for _ in range(201)]
    with gzip.GzipFile(os.path.join(HERE, "pd_coarse_snapshot_head.csv.gz"), "wb", mtime=0) as g:
        g.write("".join(head).encode())


def run_examples(reference):
    """Copies the example cases and runs the reference's CLI on each, in a scratch directory
    that is removed afterwards; the outputs are stored gzipped."""
    import subprocess
    import tempfile
    src = os.path.join(reference, "examples")
    names = sorted(n for n in os.listdir(src) if n.endswith(".json"))
    os.makedirs(os.path.join(HERE, "examples"), exist_ok=True)
    for name in names:
        shutil.copyfile(os.path.join(src, name), os.path.join(HERE, "examples", name))
    shutil.copyfile(os.path.join(reference, "configs", "elastic.json"),
                    os.path.join(HERE, "configs", "elastic.json"))
    exe = os.path.join(ROOT, "oracle", "_ref", "vumat_pd_run")
    scratch = tempfile.mkdtemp(dir=HERE, prefix=".examples_")
    try:
        shutil.copytree(os.path.join(HERE, "examples"), os.path.join(scratch, "examples"))
        shutil.copytree(os.path.join(HERE, "configs"), os.path.join(scratch, "configs"))
        for name in names:
            subprocess.run([exe, os.path.join("examples", name)], cwd=scratch, check=True,
                           stdout=subprocess.DEVNULL)
            case = name[:-5]
            out = os.path.join(scratch, "examples", "output", case)
            dst = os.path.join(HERE, "example_outputs", case)
            os.makedirs(dst, exist_ok=True)
            for f in sorted(os.listdir(out)):
                with open(os.path.join(out, f), "rb") as a, \
                        gzip.GzipFile(os.path.join(dst, f + ".gz"), "wb", mtime=0) as g:
                    g.write(a.read())
    finally:
        shutil.rmtree(scratch)


CONFIG3_SLAB_STEPS = 160
CONFIG3_SLAB_STRIDE = 13


def config3_slab():
    """The reference library (compiled into oracle/_ref) on a slab of the config-3 bar."""
    import oracle as O
    from vpd.case import tensile_bar
    case = tensile_bar(3, nx=24, precision=0)
    sim = O.RefSim(case)
    diag = sim.step(CONFIG3_SLAB_STEPS)
    pick = np.arange(0, sim.n_points, CONFIG3_SLAB_STRIDE)
    sigma = sim.get("stress_corotational")[pick][:, [0, 4, 8, 1, 5, 2]]
    np.savez_compressed(os.path.join(HERE, "ref_config3_slab.npz"), diag=diag,
                        damage_index=sim.get("damage_index")[:, 0],
                        stride=CONFIG3_SLAB_STRIDE,
                        displacement=sim.get("displacement")[pick],
                        stress_corotational6=sigma, state=sim.get("state")[pick][:, [1, 5]])
    sim.close()


def archived_cases(reference):
    """The archived PD runs and the FEM reference, reduced to what the analysis metrics read."""
    sys.path.insert(0, os.path.join(ROOT, "vumat-pd_b200"))
    from vpd.metrics import COMMON_TIMES, interpolate_nodes, read_csv, sample_coordinates
    import json
    raw = os.path.join(reference, "benchmarks", "tensile3d", "raw")
    coords = sample_coordinates()
    out = {}
    fem_ts = read_csv(os.path.join(raw, "fem_reference", "timeseries.csv.gz"))
    fem_nodes = read_csv(os.path.join(raw, "fem_reference", "final_nodes.csv.gz"))
    out["fem_reference_stress"] = np.interp(COMMON_TIMES, fem_ts["time_ms"],
                                            fem_ts["average_axial_stress_MPa"])
    out["fem_reference_final_stress"] = fem_ts["average_axial_stress_MPa"][-1]
    out["fem_reference_max_eqps"] = fem_ts["max_eqps"][-1]
    out["fem_reference_u"] = interpolate_nodes(fem_nodes, coords)
    names = sorted(n for n in os.listdir(raw) if n.startswith("pd_"))
    for name in names:
        ts = read_csv(os.path.join(raw, name, "timeseries.csv.gz"))
        cols = [k for k in ts]
        out[f"{name}_timeseries"] = np.stack([ts[k] for k in cols], 1)
        out[f"{name}_columns"] = np.array(cols)
        snap = read_csv(os.path.join(raw, name, "field_snapshots.csv.gz"))
        out[f"{name}_u"] = interpolate_nodes(snap, coords)
        with open(os.path.join(raw, name, "metadata.json")) as f:
            meta = json.load(f)
        m = meta["materials"][0]
        out[f"{name}_summary"] = np.array([m["maxEqps"], m["finalReaction_N"],
                                           m["finalEnergyError"], m["earlyElasticSlope_MPa"]])
    np.savez_compressed(os.path.join(HERE, "archived_pd_cases.npz"), **out)
    with open(os.path.join(reference, "benchmarks", "tensile3d", "expected", "analysis.json")) as f:
        expected = json.load(f)["metrics"]
    with open(os.path.join(HERE, "expected_pd_metrics.json"), "w") as f:
        json.dump({k: v for k, v in expected.items() if k.startswith("pd_")}, f, indent=1,
                  sort_keys=True)
        f.write("\n")


def main(reference):
    copy_cases(reference)
    import oracle as O
    from vpd.case import Case, REFERENCE_JC_PROPS, tensile_bar

    raw = os.path.join(reference, "benchmarks", "tensile3d", "raw", "pd_coarse")
    shutil.copyfile(os.path.join(raw, "timeseries.csv.gz"),
                    os.path.join(HERE, "pd_coarse_timeseries.csv.gz"))
    with gzip.open(os.path.join(raw, "field_snapshots.csv.gz"), "rt") as f:
        rows = list(csv.reader(f))
    header, body = rows[0], rows[1:]
    cols = {name: i for i, name in enumerate(header)}
    last = [r for r in body if int(r[cols["step"]]) == 4800]
    last.sort(key=lambda r: int(r[cols["particle"]]))

    def column(name):
        return np.array([float(r[cols[name]]) for r in last])

    np.savez_compressed(
        os.path.join(HERE, "pd_coarse_snapshot.npz"),
        displacement=np.stack([column("ux_mm"), column("uy_mm"), column("uz_mm")], 1),
        velocity=np.stack([column("vx_mm_per_ms"), column("vy_mm_per_ms"), column("vz_mm_per_ms")], 1),
        axial_strain=column("axial_strain"), axial_stress=column("axial_stress_MPa"),
        eqps=column("eqps"))

    # neighbour lists of the reference library on a jittered lattice
    small = Case(name="jittered", nx=17, ny=9, nz=5, spacing=1.25, horizon=3.015 * 1.25,
                 dt=1e-5, steps=1, density=0.0078, props=REFERENCE_JC_PROPS, jitter=0.05,
                 jitter_seed=11, grip_velocity=1.0, ramp_time=1e-3)
    sim = O.RefSim(small)
    pos = sim.get("position")
    row_ptr, col = sim.neighbors()
    np.savez_compressed(os.path.join(HERE, "ref_neighbors_jittered.npz"), positions=pos,
                        horizon=small.horizon, row_ptr=row_ptr, col=col)
    sim.close()

    # the reference library on the 40x10x10 bar with jitter and damage
    bar = tensile_bar(1, jitter=0.05, jitter_seed=7, damage_mode=1, damage_initiation=0.004)
    sim = O.RefSim(bar)
    diag = sim.step(300)
    np.savez_compressed(os.path.join(HERE, "ref_tensile_bar_1.npz"), diag=diag,
                        displacement=sim.get("displacement"),
                        stress_corotational=sim.get("stress_corotational"),
                        state=sim.get("state"), damage_index=sim.get("damage_index"))
    sim.close()

    # one plastic JC step (jc_thermal_units_test.cpp:9-20) in both heat-unit conventions
    out = {}
    for tag, w2h in (("legacy", 1.0), ("scaled", 1.0e6)):
        props = np.array(REFERENCE_JC_PROPS[:13] + (w2h,))
        first = O.vumat_block(O.oracle_lib(), props, 2.5e-5, np.zeros((1, 6)), np.zeros((1, 6)),
                              np.zeros((1, 6)), np.array([293.0]), np.zeros(1), np.zeros(1))
        inc = np.zeros((1, 6))
        inc[0, 0] = 400 * 2.5e-5
        second = O.vumat_block(O.oracle_lib(), props, 2.5e-5, inc, first["stress"], first["state"],
                               first["temperature"], first["energy_internal"],
                               first["energy_inelastic"])
        for k, v in second.items():
            out[f"{tag}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "ref_jc_thermal.npz"), **out)
    config3_slab()
    archived_cases(reference)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if not args or not os.path.isdir(os.path.join(args[0], "src")):
        sys.exit("usage: make_golden.py REFERENCE_CHECKOUT [--cases-only | --examples]")
    ref = args[0]
    if "--cases-only" in sys.argv:
        copy_cases(ref)
    elif "--examples" in sys.argv:
        run_examples(ref)
    elif "--config3" in sys.argv:
        config3_slab()
    elif "--archived" in sys.argv:
        archived_cases(ref)
    else:
        main(ref)
        run_examples(ref)
