"""Golden fixtures (tests/golden/cycles.json, written by
tests/golden/make_golden.py from bismit's own kernels compiled for the CPU):
the SHA-256 of the whole state slab after every cycle, from seeded states.
The C restatement must reproduce them on the CPU and the CUDA paths on the
GPU, with no reference code at test time."""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle  # noqa: E402
from make_golden import CASES, initial_state  # noqa: E402

GOLD = json.load(open(os.path.join(HERE, "golden", "cycles.json")))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", sorted(CASES))
def test_restatement_reproduces_reference_digests(name):
    g = GOLD[name]
    plan, desc, slab, frames = initial_state(name)
    assert int(plan.slab_bytes) == g["slab_bytes"] and int(plan.n_syns_total) == g["n_syns"]
    assert sha(slab) == g["initial_sha256"]
    for c in range(g["cycles"]):
        oracle.run(plan, slab, frames[c:c + 1], 1, c)
        assert sha(slab) == g["after_cycle_sha256"][c], "cycle %d" % c


@pytest.mark.gpu
@pytest.mark.parametrize("plain", [False, True], ids=["fused", "plain"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_device_reproduces_reference_digests(name, plain):
    from bismit_b200 import _ffi as F, cortex
    g = GOLD[name]
    plan, desc, slab, frames = initial_state(name)
    if plain:
        desc.exec_path = F.BM_PATH_PLAIN
    ctx = cortex._Ctx(0)
    area = cortex.CorticalArea(ctx, desc, g["growth_seed"])
    area.write_slab(slab)
    area.set_cycle(0)
    for c in range(g["cycles"]):
        area.write_input(frames[c])
        area.cycle(1)
        assert sha(area.read_slab()) == g["after_cycle_sha256"][c], "cycle %d" % c
    area.close()
    ctx.close()
