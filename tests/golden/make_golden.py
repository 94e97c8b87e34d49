"""Writes the golden fixtures of this directory from bismit's own kernels.

The fixtures pin the cycle to the reference: bismit's cl/*.cl compiled for
the CPU (oracle/_ref, built by `make -C oracle ref` from a bismit checkout)
run each case from a seeded, scrambled state for a few cycles with learning
on. The initial state and the frames are reproducible from their seeds
(seeded growth, scramble and frames are this repository's code), so each
case stores the seeds, the plan's slab size and synapse count, the SHA-256
of the initial slab (a changed growth or layout is caught rather than
compared) and the SHA-256 of the whole slab after every cycle. Run from the
repository root:

    python tests/golden/make_golden.py

Needs oracle/_ref; the fixtures it writes are what the tests read, with no
reference at test time.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from bismit_b200 import configs, map as M, plan_of  # noqa: E402
from helpers import scramble  # noqa: E402

# name: (layer maps, growth seed, scramble seed, frame seed, cycles, input activity)
CASES = {
    "testbed_16": (lambda: configs.testbed_area(16), 3, 11, 5, 6, 0.05),
    "mixed_24": (lambda: configs.mixed_area(24, 32), 4, 12, 6, 6, 0.05),
    "instance_32": (lambda: configs.instance_area(32, 2, 8, 32), 5, 13, 7, 6, 0.03),
}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def initial_state(name):
    """(plan, desc, initial slab, frames) of case `name`, from its seeds."""
    build, gseed, sseed, fseed, cycles, active = CASES[name]
    lmaps, areas = build()
    desc = M.area_desc("v1", lmaps, areas, configs.bench_settings())
    plan = plan_of(desc, gseed)
    slab = np.zeros(int(plan.slab_bytes), np.uint8)
    oracle.grow(plan, slab, gseed, desc.init_flags)
    scramble(plan, slab, sseed)
    frames = configs.frames(cycles, int(plan.inputs[0].len), active, fseed)
    return plan, desc, slab, frames


def main():
    if oracle.load_ref() is None:
        raise SystemExit("oracle/_ref is not built: run `make -C oracle ref` with a bismit checkout")
    out = {}
    for name, (_b, gseed, sseed, fseed, cycles, active) in CASES.items():
        plan, desc, slab, frames = initial_state(name)
        rec = {"growth_seed": gseed, "scramble_seed": sseed, "frame_seed": fseed, "cycles": cycles,
               "active": active, "slab_bytes": int(plan.slab_bytes), "n_syns": int(plan.n_syns_total),
               "initial_sha256": sha(slab), "after_cycle_sha256": []}
        for c in range(cycles):
            oracle.run(plan, slab, frames[c:c + 1], 1, c, impl="ref")
            rec["after_cycle_sha256"].append(sha(slab))
        out[name] = rec
        print(name, plan.slab_bytes)
    with open(os.path.join(HERE, "cycles.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
