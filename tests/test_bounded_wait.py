"""The give-up path of the tuft kernels' bounded waits, made to run on the
GPU without a fault.

A test hook (bm_area_inject_stall) makes block 0's copy lane of every tiled
tuft launch withhold one shared-memory stage: it neither copies nor arms
that stage's barrier, so the consumers' wait for it can only run out. With
the wait limit at 1 ms (bm_area_set_wait_limit) the consumers give up, set
error bit 0, and the kernel lets its own copies land and returns. The host
then sees the bits (bm_area_device_errors), further cycling calls are
refused with BM_ERR_TIMEOUT, and after the caller restores a state and
clears the bits the area cycles bit-exactly again. Every wait involved stays
bounded: nothing traps, asserts or hangs. bismit has no counterpart (it
panics on errors, src/cortex/cortex.rs:111).
"""
import numpy as np
import pytest

import oracle
from bismit_b200 import _ffi as F, configs, cortex, map as M
from helpers import diff_report, frames_for, settings_for, desc_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = cortex._Ctx(0)
    yield c
    c.close()


def _tiled(area):
    p = area.plan
    return [(i, t) for i in range(p.n_layers) for t in range(p.layers[i].n_tufts) if area.tuft_form(i, t)["tiled"]]


def _check_recovers(area, slab0, fr, cycles=3):
    area.clear_errors()
    assert area.device_errors() == 0
    area.write_slab(slab0)
    area.set_cycle(0)
    ora = slab0.copy()
    for k in range(cycles):
        area.write_input(fr[k])
        area.cycle(1)
        oracle.run(area.plan, ora, fr[k:k + 1], 1, start_cycle=k)
        dev = area.read_slab()
        assert np.array_equal(dev, ora), "cycle %d after recovery:\n%s" % (k, diff_report(area.plan, dev, ora))
    assert area.device_errors() == 0


@pytest.mark.parametrize("stage", [1, 2])
def test_withheld_stage_gives_up_and_reports(ctx, stage):
    area = cortex.CorticalArea(ctx, desc_of("area_64", settings_for()), 7)
    assert len(_tiled(area)) >= 2
    slab0 = area.read_slab()
    fr = frames_for(area.plan, 3, 5, 0.05)
    area.set_wait_limit(1000)
    area.inject_stall(stage)
    area.write_input(fr[0])
    area.cycle(1)                       # enqueues; the kernels give up on their own
    ctx.synchronize()
    assert area.device_errors() == 1
    with pytest.raises(F.BismitError) as e:
        area.cycle(1)
    assert e.value.code == F.BM_ERR_TIMEOUT
    assert area.cycle_count() == 1      # the refused call enqueued nothing
    area.inject_stall(0)
    area.set_wait_limit(0)
    _check_recovers(area, slab0, fr)
    area.close()


def test_withheld_stage_in_a_batch(ctx):
    """In a graph-replayed batch the stalled area's bits are set, the other
    area's are not, the batch refuses further cycles, and once the bits are
    cleared and the states restored both areas match cycling alone."""
    descs = [M.area_desc("v1", *configs.instance_area(side, 2, 16, 32), configs.bench_settings()) for side in (48, 64)]
    areas = [cortex.CorticalArea(ctx, d, 3 + k) for k, d in enumerate(descs)]
    slabs = [a.read_slab() for a in areas]
    frames = [configs.frames(3, a.input_len(), 0.03, 20 + k) for k, a in enumerate(areas)]
    batch = cortex.Batch(ctx, areas)
    for a in areas:
        a.set_wait_limit(1000)
    areas[1].inject_stall(1)
    for k, a in enumerate(areas):
        a.write_input(frames[k][0])
    batch.cycle(1)
    ctx.synchronize()
    assert areas[0].device_errors() == 0
    assert areas[1].device_errors() == 1
    with pytest.raises(F.BismitError) as e:
        batch.cycle(1)
    assert e.value.code == F.BM_ERR_TIMEOUT
    areas[1].inject_stall(0)
    for k, a in enumerate(areas):
        a.set_wait_limit(0)
        a.clear_errors()
        a.write_slab(slabs[k])
        a.set_cycle(0)
    ora = [s.copy() for s in slabs]
    for c in range(3):
        for k, a in enumerate(areas):
            a.write_input(frames[k][c])
        batch.cycle(1)
        for k, a in enumerate(areas):
            oracle.run(a.plan, ora[k], frames[k][c:c + 1], 1, start_cycle=c)
            dev = a.read_slab()
            assert np.array_equal(dev, ora[k]), "cycle %d area %d:\n%s" % (c, k, diff_report(a.plan, dev, ora[k]))
    assert batch.device_errors() == 0
    batch.close()
    for a in areas:
        a.close()


def test_wait_limit_alone_changes_nothing(ctx):
    """A short limit with nothing withheld: no wait runs out on a healthy
    ring, so the results are the oracle's."""
    area = cortex.CorticalArea(ctx, desc_of("area_48_deep", settings_for()), 9)
    slab0 = area.read_slab()
    fr = frames_for(area.plan, 3, 6, 0.05)
    area.set_wait_limit(50000)
    _check_recovers(area, slab0, fr)
    area.close()
