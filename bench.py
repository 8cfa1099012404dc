#!/usr/bin/env python
"""Throughput of the correspondence-PD explicit increment on the 1M-point steel bar.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl vpd|reference]

Workload: the 400x50x50 jittered Johnson-Cook tensile bar (1,000,000 points, horizon
4.015 h, about 238 bonds per point, critical-stretch damage, grips pulled at 5 m/s). A step
is one explicit increment of the whole bar. One process per GPU (torchrun); the path does not
shard across GPUs, so N GPUs run N independent replicas ("replicas only") and the value is
the sum of their particle-steps/s, timed as the max over ranks.

Printed JSON line (rank 0):
  value        particle-steps/s, device time (CUDA events on the library's stream) of K
               increments after W warm-up increments, inputs resident in HBM
  e2e          the same K increments through the C ABI as a host driver runs them: the case
               created from host position/volume arrays, one vpd_step call per increment
               returning its timeseries row to host memory, and the final snapshot fields
               copied back; host wall clock
  roofline     the dominant kernel's algorithmic bytes / its CUDA-event time vs the measured
               HBM copy bandwidth; traffic from the ncu capture summarised in profiles/
  cpu_baseline the reference library (compiled from its sources into oracle/_ref) on a
               100k-point slab of the same bar, all host threads
--impl reference prints the reference library's own line for the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "vumat-pd_b200"))

METRIC = "particle-steps/s at 1M pts: surrogate-PD vs plain-PD at <=0.5% stress NRMSE"
UNIT = "particle-steps/s"
SAMPLE_NX = 40  # CPU sample: 40x50x50 slab of the bar


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="vpd", choices=("vpd", "reference"))
    p.add_argument("--nx", type=int, default=400, help="bar length in lattice planes")
    p.add_argument("--plastic-preload", type=int, default=2000,
                   help="extra measurement after this many increments (0 disables)")
    p.add_argument("--cpu-steps", type=int, default=12)
    return p.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region (clocks, throttle reasons)."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        lines = [l.strip() for l in self.file.read().splitlines() if l.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(nb, damage):
    """Bytes each kernel must move per point per increment (FP64 state): reads and writes of
    the per-point arrays it owns plus one 4-byte neighbour index per bond (and one bit per bond
    read and written when damage is on)."""
    d = 0.25 * nb if damage else 0.0
    return {
        # x,y,z,V + u of the point, K^-1, F written, neighbour indices, broken-bond bits
        "deformation": 32 + 24 + 72 + 72 + 4 * nb + d,
        # F, F_n, V_n, R_n, K^-1, E, sigma, state, energies, volume, window weight read;
        # F_n, V_n, R_n, E, sigma, state, energies, force map written
        "material": 72 * 5 + 48 * 3 + 16 + 16 + 72 * 3 + 48 * 3 + 16 + 72,
        # x,y,z,V, M, u, v, a, flags read; u, v, a, f written; indices and bits
        "force": 32 + 72 + 24 + 48 + 1 + 24 + 48 + 24 + 4 * nb + 0.125 * nb,
    }


def ncu_traffic():
    """DRAM bytes per point per kernel launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


def cpu_reference(steps, warmup):
    """The reference library (oracle/_ref, all host threads) on the 100k-point slab."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from vpd.case import tensile_bar
    case = tensile_bar(3, nx=SAMPLE_NX, precision=0)
    sim = O.RefSim(case)
    sim.step(warmup)
    t0 = time.perf_counter()
    sim.step(steps)
    dt = time.perf_counter() - t0
    n = sim.n_points
    stages = sim.stage_seconds()
    sim.close()
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": n * steps / dt, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{SAMPLE_NX}x50x50 slab of the bar ({n} points, same horizon, jitter, "
                      f"damage), increments {warmup + 1}-{warmup + steps} from rest",
            "stage_seconds": {k: round(v, 3) for k, v in stages.items()}}


def run_reference(args, world, rank):
    if rank != 0:
        return
    base = cpu_reference(args.steps, args.warmup)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "tensile_bar_3 (400x50x50 jittered steel JC bar), CPU sample",
                   "sample": base["sample"]},
        "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def run_gpu(args, world, rank, local):
    import numpy as np
    import torch
    import vpd
    from vpd.case import tensile_bar

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    case = tensile_bar(3, nx=args.nx, precision=0)
    K, W = args.steps, args.warmup
    sim = vpd.Simulation(case)
    n, nb = sim.n_points, sim.n_bonds / sim.n_points
    sim.step(W, diagnostics=False)
    barrier()
    clocks = ClockSampler(local)
    rows = sim.step(K, diagnostics=True)
    barrier()
    clock = clocks.stop()
    ms = max_over_ranks(sim.last_step_ms())
    value = world * n * K / (ms * 1e-3)
    finite = bool(rows[-1, vpd.DIAG["finite"]] == 1.0)

    # per-kernel CUDA-event times (separate launches on the library stream)
    stages = sim.profile_stages(5)
    sim.close()

    # end to end through the C ABI with host buffers
    positions = vpd.Simulation(case.replace(nx=args.nx))
    host_pos, host_vol = positions.field("position"), positions.field("volume")[:, 0].copy()
    positions.close()
    barrier()
    t0 = time.perf_counter()
    e2e_sim = vpd.Simulation(case, positions=host_pos, volumes=host_vol)
    for _ in range(K):
        e2e_sim.step(1, diagnostics=True)
    snap = [e2e_sim.field(f) for f in ("displacement", "velocity", "stress_spatial", "state")]
    e2e_s = time.perf_counter() - t0
    e2e_sim.close()
    e2e_s = max_over_ranks(e2e_s)
    h2d = host_pos.nbytes + host_vol.nbytes
    d2h = sum(a.nbytes for a in snap) + K * len(vpd.DIAG_COLUMNS) * 8

    # the plastic regime: after a preload the JC return map runs at most points
    plastic = None
    if args.plastic_preload > 0:
        ps = vpd.Simulation(case)
        ps.step(args.plastic_preload, diagnostics=False)
        r = ps.step(K, diagnostics=True)
        pms = max_over_ranks(ps.last_step_ms())
        plastic = {"start_increment": args.plastic_preload + 1,
                   "value": world * n * K / (pms * 1e-3), "ms_per_step": pms / K,
                   "max_eqps": float(r[-1, vpd.DIAG["max_eqps"]])}
        ps.close()

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peak, peak_kind = measured_peaks()
    alg = algorithmic_bytes(nb, case.damage_mode == 1)
    dominant = max(stages, key=stages.get)
    achieved = alg[dominant] * n / (stages[dominant] * 1e-3) / 1e9
    traffic = ncu_traffic()
    tr = None
    if traffic and dominant in traffic.get("bytes_per_point", {}):
        tr = traffic["bytes_per_point"][dominant] * n
    step_bytes = sum(alg.values()) * n
    cpu = cpu_reference(args.cpu_steps, 2)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "tensile_bar_3: 400x50x50 jittered (+-0.05 h) steel Johnson-Cook "
                               "bar, horizon 4.015 h, critical stretch 0.02, grips 5 m/s",
                   "points": n, "bonds_per_point": round(nb, 2), "precision": "fp64 plain",
                   "material": "device Johnson-Cook VUMAT",
                   "increments": f"{W + 1}-{W + K} from rest",
                   "l2": "working set ~4 GB > 126 MB L2, no flush needed",
                   "parallelism": f"replicas x{world}"},
        "modes": {"plain_fp64": {"value": value, "stress_nrmse_vs_fp64": 0.0}},
        "plastic_regime": plastic,
        "stage_ms": {k: round(v, 4) for k, v in stages.items()},
        "step_roofline": {"algorithmic_bytes": step_bytes,
                          "achieved_gbs": step_bytes / (ms / K * 1e-3) / 1e9,
                          "frac": step_bytes / (ms / K * 1e-3) / 1e9 / peak},
        "roofline": {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": tr, "algorithmic_bytes": alg[dominant] * n},
        "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": world * n * K / e2e_s * 1.0, "unit": UNIT,
                "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
                "includes": "vpd_create from host arrays (neighbour search, K^-1), K increments "
                            "from rest one call each with their rows read back, final snapshot "
                            "download"},
        "gpu_launches": 3 * K,
        "clocks": clock,
        "finite": finite,
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def main():
    args = parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_gpu(args, world, rank, local)


if __name__ == "__main__":
    main()
