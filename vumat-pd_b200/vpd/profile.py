"""Per-stage timing of the increment on one tensile-bar workload (CUDA events on the handle's
stream), for profiling runs:

    python -m vpd.profile --config 3 --nx 100 --precision mixed --warm 2 --steps 4

Prints one JSON line: points, bonds, layout words, ms per increment over --steps graph
increments, and the four stage times (deformation, material, force, integrate) averaged over
--stage-steps separately launched increments. Under a kernel profiler, --steps 0 and
--stage-steps 1 keep the number of launches small.

--save-checkpoint PATH writes the state after the --warm increments (and the network, for the
surrogate, to PATH.net.npz); --load-checkpoint PATH starts from such a state instead of
running --warm increments, so a profiler run of one increment in plastic flow has only the set-up
launches before it:

    python -m vpd.profile --nx 100 --warm 700 --steps 0 --stage-steps 0 --save-checkpoint /tmp/ck
    ncu ... python -m vpd.profile --nx 100 --load-checkpoint /tmp/ck --steps 0 --stage-steps 1
"""
from __future__ import annotations

import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import vpd  # noqa: E402
from vpd.case import tensile_bar  # noqa: E402


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--nx", type=int, default=100)
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    ap.add_argument("--no-damage", action="store_true")
    ap.add_argument("--warm", type=int, default=2, help="untimed increments first")
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--stage-steps", type=int, default=3)
    ap.add_argument("--surrogate", choices=("network", "hybrid", "warm_start"),
                    help="material_mode surrogate with this guess (default: the VUMAT)")
    ap.add_argument("--newton-steps", type=int, default=2)
    ap.add_argument("--train-samples", type=int, default=400_000,
                    help="increments for the network trained before the run")
    ap.add_argument("--train-epochs", type=int, default=4)
    ap.add_argument("--save-checkpoint", help="write the state after --warm increments here")
    ap.add_argument("--load-checkpoint", help="start from this state (instead of --warm)")
    a = ap.parse_args(argv)
    over = {"nx": a.nx, "precision": 1 if a.precision == "mixed" else 0}
    if a.no_damage:
        over["damage_mode"] = 0
    weights = (None, None)
    if a.surrogate:
        over["material_mode"] = 1
        if a.surrogate != "warm_start":
            if a.load_checkpoint:
                import numpy as np
                net = np.load(a.load_checkpoint + ".net.npz")
                weights = (net["w"], net["b"])
            else:
                w, b, _ = vpd.train_surrogate(tensile_bar(a.config).props, samples=a.train_samples,
                                              epochs=a.train_epochs)
                weights = (w, b)
                if a.save_checkpoint:
                    import numpy as np
                    np.savez(a.save_checkpoint + ".net.npz", w=w, b=b)
    case = tensile_bar(a.config, **over)
    with vpd.Simulation(case) as sim:
        if a.surrogate:
            sim.set_surrogate(*weights, guess=a.surrogate, newton_steps=a.newton_steps)
        if a.load_checkpoint:
            with open(a.load_checkpoint, "rb") as f:
                sim.restore(f.read())
        elif a.warm:
            sim.step(a.warm, diagnostics=False)
        if a.save_checkpoint:
            with open(a.save_checkpoint, "wb") as f:
                f.write(sim.checkpoint())
        ms = None
        if a.steps:
            sim.step(a.steps, diagnostics=False)
            ms = sim.last_step_ms() / a.steps
        stages = sim.profile_stages(a.stage_steps) if a.stage_steps else {}
        print(json.dumps({"config": a.config, "nx": a.nx, "precision": a.precision,
                          "damage": not a.no_damage, "surrogate": a.surrogate,
                          "points": sim.n_points, "bonds": sim.n_bonds,
                          "layout_words": sim.layout_words, "ms_per_increment": ms,
                          "stage_ms": stages}))


if __name__ == "__main__":
    main()
