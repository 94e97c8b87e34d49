"""Batched cycling (bm_batch_*): several areas of one layer map and uneven
sizes advanced together must leave every area with exactly the bytes it has
after cycling alone, and those bytes must match the oracle.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from bismit_b200 import _ffi as F, configs, cortex, map as M
from helpers import buffers, diff_report, scramble

# (side, depth, distal dens, distal syns): a small spread of the batched
# workload's shapes, proximal 1 x 1 tufts included (the unfused sub-stages).
SMALL = [(32, 1, 8, 16), (48, 2, 16, 32), (64, 1, 8, 64), (40, 3, 16, 16)]


def _desc(side, depth, dens, syns, settings=None):
    lmaps, areas = configs.instance_area(side, depth, dens, syns)
    return M.area_desc("v1", lmaps, areas, settings or configs.bench_settings())


def _deep_desc(side):
    """The area_48_deep layer map (fused proximal 4 x 16 tufts) on other grids."""
    lmaps, areas = configs.benchmark_area(side, 32, 2, 4, 16, 3)
    return M.area_desc("v1", lmaps, areas, configs.bench_settings())


def _frames(area, n, seed):
    return configs.frames(n, int(area.plan.inputs[0].len), 0.03, seed)


def _pairs(ctx, descs, seed=5):
    """Twin areas per descriptor: one to batch, one to cycle alone, from the
    same scrambled state."""
    batched, alone = [], []
    for k, d in enumerate(descs):
        a = cortex.CorticalArea(ctx, d, seed + k)
        b = cortex.CorticalArea(ctx, d, seed + k)
        slab = a.read_slab()
        scramble(a.plan, slab, 100 + k)
        a.write_slab(slab)
        b.write_slab(slab)
        a.set_cycle(0)
        b.set_cycle(0)
        batched.append(a)
        alone.append(b)
    return batched, alone


def _check_equal(batched, alone, when):
    for k, (a, b) in enumerate(zip(batched, alone)):
        x, y = a.read_slab(), b.read_slab()
        assert np.array_equal(x, y), "%s, area %d:\n%s" % (when, k, diff_report(a.plan, x, y))


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [True, False], ids=["graph", "eager"])
@pytest.mark.parametrize("kind", ["instances", "deep"])
def test_batch_matches_areas_alone(graph, kind):
    ctx = cortex._Ctx(0)
    descs = [_desc(*s) for s in SMALL] if kind == "instances" else [_deep_desc(s) for s in (32, 48, 56)]
    batched, alone = _pairs(ctx, descs)
    batch = cortex.Batch(ctx, batched, graph=graph)
    fr = [_frames(a, 6, 30 + k) for k, a in enumerate(batched)]
    for c in range(6):
        for k in range(len(batched)):
            batched[k].write_input(fr[k][c])
            alone[k].write_input(fr[k][c])
            alone[k].cycle(1)
        batch.cycle(1)
        _check_equal(batched, alone, "cycle %d" % c)
    assert batch.device_errors() == 0
    assert all(a.cycle_count() == 6 for a in batched)
    batch.close()
    for a in batched + alone:
        a.close()
    ctx.close()


@pytest.mark.gpu
def test_batch_frames_from_device_match_areas_alone():
    import torch
    ctx = cortex._Ctx(0)
    batched, alone = _pairs(ctx, [_desc(*s) for s in SMALL])
    batch = cortex.Batch(ctx, batched)
    n = 5
    fr = [_frames(a, n, 60 + k) for k, a in enumerate(batched)]
    packed = batch.pack_frames(fr)
    assert packed.shape == (n, batch.frame_bytes())
    dev = torch.from_numpy(packed).to("cuda:0")
    torch.cuda.synchronize()
    batch.cycle_frames_device(dev.data_ptr(), n)
    ctx.synchronize()
    for c in range(n):
        for k in range(len(alone)):
            alone[k].write_input(fr[k][c])
            alone[k].cycle(1)
    _check_equal(batched, alone, "after %d device-fed cycles" % n)
    batch.close()
    for a in batched + alone:
        a.close()
    ctx.close()


def _regrowth_settings():
    s = configs.bench_settings()
    s.bits &= ~F.BM_SET_DISABLE_REGROWTH
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("regrowth", [False, True], ids=["static", "regrowth"])
def test_batch_matches_oracle(regrowth):
    """The graph-replayed batch against the oracle; with regrowth on, over
    cycles 198 to 201 (the batch's one regrowth launch for every area acts at
    cycle 200)."""
    ctx = cortex._Ctx(0)
    st = _regrowth_settings() if regrowth else None
    start = 198 if regrowth else 0
    batched, alone = _pairs(ctx, [_desc(*s, settings=st) for s in SMALL[:3]])
    for a in batched:
        a.set_cycle(start)
    batch = cortex.Batch(ctx, batched)
    ora = [a.read_slab() for a in batched]
    first = [o.copy() for o in ora]
    fr = [_frames(a, 4, 80 + k) for k, a in enumerate(batched)]
    for c in range(4):
        for k, a in enumerate(batched):
            a.write_input(fr[k][c])
        batch.cycle(1)
        for k, a in enumerate(batched):
            oracle.run(a.plan, ora[k], fr[k][c:c + 1], 1, start_cycle=start + c)
            dev = a.read_slab()
            assert np.array_equal(dev, ora[k]), "cycle %d area %d:\n%s" % (start + c, k, diff_report(a.plan, dev, ora[k]))
    if regrowth:
        for k, a in enumerate(batched):
            moved = 0
            for name, off, n in buffers(a.plan):
                if name.endswith("syn_src_col_v_offs"):
                    moved += int(np.count_nonzero(first[k][off:off + n] != ora[k][off:off + n]))
            assert moved > 0, k
    batch.close()
    for a in batched + alone:
        a.close()
    ctx.close()


@pytest.mark.gpu
def test_batch_autotune_keeps_state_and_parity(tmp_path):
    ctx = cortex._Ctx(0)
    batched, alone = _pairs(ctx, [_desc(*s) for s in SMALL])
    batch = cortex.Batch(ctx, batched)
    before = [a.read_slab() for a in batched]
    cache = str(tmp_path / "tiles.txt")
    n = batch.autotune(cache)
    assert n >= 1
    for a, s in zip(batched, before):
        assert np.array_equal(a.read_slab(), s), "autotune changed an area's state"
    rows = [l.split() for l in open(cache).read().split("\n") if l.strip()]
    assert rows and all(len(r) == 5 for r in rows), rows   # key, tile target, stages, CTAs per SM, staged
    assert all(int(r[1]) >= 4096 and int(r[2]) in (0, 2, 3) and int(r[3]) in (0, 1, 2) and int(r[4]) in (0, 1)
               for r in rows), rows
    assert batch.autotune(cache) == n   # applied from the cache
    fr = [_frames(a, 4, 90 + k) for k, a in enumerate(batched)]
    for c in range(4):
        for k in range(len(batched)):
            batched[k].write_input(fr[k][c])
            alone[k].write_input(fr[k][c])
            alone[k].cycle(1)
        batch.cycle(1)
    _check_equal(batched, alone, "after autotune")
    batch.close()
    for a in batched + alone:
        a.close()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("stages,ctas,staged", [(2, 1, 0), (3, 2, 1), (2, 0, 1), (0, 1, 0)])
def test_batch_launch_shapes_from_cache(tmp_path, stages, ctas, staged):
    """Every launch shape the autotuner may choose (ring stages, CTAs per SM,
    footprint form) leaves the batched areas equal to cycling alone: the
    shapes are forced through a cache file written with the tuned keys."""
    ctx = cortex._Ctx(0)
    descs = [_desc(*s) for s in SMALL] + [_deep_desc(64)]
    batched, alone = _pairs(ctx, descs, seed=31)
    batch = cortex.Batch(ctx, batched)
    cache = str(tmp_path / "tiles.txt")
    batch.autotune(cache)
    rows = [l.split() for l in open(cache).read().split("\n") if l.strip()]
    assert rows
    with open(cache, "w") as f:
        for r in rows:
            f.write("%s %s %d %d %d\n" % (r[0], r[1], stages, ctas, staged))
    batch.close()
    for a in batched:   # autotuning restored the state it touched
        a.set_cycle(0)
    batch = cortex.Batch(ctx, batched)
    assert batch.autotune(cache) == len(rows)
    tma = {area.tuft_form(i, t)["footprint_tma"] for area in batched for i in range(area.plan.n_layers)
           for t in range(area.plan.layers[i].n_tufts) if area.tuft_form(i, t)["tiled"]}
    # Side 40 rows are not a multiple of 16 bytes: with tensor boxes allowed,
    # one launch mixes boxed and staged footprints.
    assert tma == ({False} if staged else {False, True}), tma
    fr = [_frames(a, 3, 70 + k) for k, a in enumerate(batched)]
    for c in range(3):
        for k in range(len(batched)):
            batched[k].write_input(fr[k][c])
            alone[k].write_input(fr[k][c])
            alone[k].cycle(1)
        batch.cycle(1)
        _check_equal(batched, alone, "stages %d, CTAs per SM %d, staged %d, cycle %d" % (stages, ctas, staged, c))
    assert batch.device_errors() == 0
    batch.close()
    for a in batched + alone:
        a.close()
    ctx.close()


@pytest.mark.gpu
def test_batch_groups_areas_with_different_programs():
    """Areas whose stage programs differ (learning off in one, another layer
    map in another) share one schedule; each still ends with its bytes from
    cycling alone."""
    ctx = cortex._Ctx(0)
    descs = [_desc(32, 1, 8, 16), _desc(48, 2, 8, 32, configs.bench_settings().disable_learning()),
             _desc(40, 1, 16, 16), _deep_desc(32)]
    batched, alone = _pairs(ctx, descs)
    batch = cortex.Batch(ctx, batched)
    fr = [_frames(a, 3, 70 + k) for k, a in enumerate(batched)]
    for c in range(3):
        for k in range(len(batched)):
            batched[k].write_input(fr[k][c])
            alone[k].write_input(fr[k][c])
            alone[k].cycle(1)
        batch.cycle(1)
        _check_equal(batched, alone, "cycle %d" % c)
    batch.close()
    for a in batched + alone:
        a.close()
    ctx.close()


def test_batch_instances_are_seeded_and_in_range():
    x = configs.batch_instances(64, 0)
    assert x == configs.batch_instances(64, 0)
    assert x != configs.batch_instances(64, 1)
    for side, depth, dens, syns, act in x:
        assert side in range(32, 193, 16) and 1 <= depth <= 4
        assert dens in (8, 16) and syns in (16, 32, 64) and 0.01 <= act <= 0.04
    # The first instance does not depend on how many are drawn.
    assert configs.batch_instances(1, 0)[0] == x[0]


@pytest.mark.gpu
def test_batch_with_smoothers_matches_oracle():
    """Areas with ActivitySmoother control layers (each area's own six lattice
    launches inside the batched cycle) against the oracle."""
    ctx = cortex._Ctx(0)
    descs = [M.area_desc("v1", *configs.smoother_area(side, 3, 2), configs.bench_settings()) for side in (40, 56)]
    batched, alone = _pairs(ctx, descs)
    batch = cortex.Batch(ctx, batched)
    ora = [a.read_slab() for a in batched]
    fr = [_frames(a, 3, 90 + k) for k, a in enumerate(batched)]
    for c in range(3):
        for k, a in enumerate(batched):
            a.write_input(fr[k][c])
        batch.cycle(1)
        for k, a in enumerate(batched):
            oracle.run(a.plan, ora[k], fr[k][c:c + 1], 1, start_cycle=c)
            dev = a.read_slab()
            assert np.array_equal(dev, ora[k]), "cycle %d area %d:\n%s" % (c, k, diff_report(a.plan, dev, ora[k]))
    batch.close()
    for a in batched + alone:
        a.close()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("device_frames", [False, True], ids=["host_frames", "device_frames"])
def test_batch_with_filters_matches_oracle(device_frames):
    """Areas with retina filter chains (one filter on a 48-wide input, two on
    a two-slice 64-wide one, three on a 32-wide source scaled into a 64-wide
    area) and one without, batched, with frames written per area or taken
    from a device frame block, against the oracle."""
    import torch
    ctx = cortex._Ctx(0)
    st = configs.bench_settings()
    descs = [M.area_desc("v1", *configs.retina_area(48), st),
             M.area_desc("v1", *configs.retina_area(64, 2, 2), st),
             M.area_desc("v1", *configs.retina_area(64, 3, 1, src_side=32), st),
             _desc(*SMALL[0])]
    batched, alone = _pairs(ctx, descs)
    batch = cortex.Batch(ctx, batched)
    ora = [a.read_slab() for a in batched]
    fr = [_frames(a, 3, 70 + k) for k, a in enumerate(batched)]
    if device_frames:
        dev = torch.from_numpy(batch.pack_frames(fr)).to("cuda:0")
        torch.cuda.synchronize()
        batch.cycle_frames_device(dev.data_ptr(), 3)
    for c in range(3):
        if not device_frames:
            for k, a in enumerate(batched):
                a.write_input(fr[k][c])
            batch.cycle(1)
        for k, a in enumerate(batched):
            oracle.run(a.plan, ora[k], fr[k][c:c + 1], 1, start_cycle=c)
            if not device_frames:
                dev_slab = a.read_slab()
                assert np.array_equal(dev_slab, ora[k]), "cycle %d area %d:\n%s" % (
                    c, k, diff_report(a.plan, dev_slab, ora[k]))
    for k, a in enumerate(batched):
        dev_slab = a.read_slab()
        assert np.array_equal(dev_slab, ora[k]), "area %d:\n%s" % (k, diff_report(a.plan, dev_slab, ora[k]))
    batch.close()
    for a in batched + alone:
        a.close()
    ctx.close()


@pytest.mark.gpu
def test_destroying_an_area_first_detaches_its_batch():
    """An area destroyed before its batch leaves the batch: the batch refuses
    to cycle, and destroying it afterwards touches nothing freed."""
    ctx = cortex._Ctx(0)
    a = cortex.CorticalArea(ctx, _desc(*SMALL[0]), 3)
    b = cortex.CorticalArea(ctx, _desc(*SMALL[1]), 4)
    batch = cortex.Batch(ctx, [a, b])
    batch.cycle(1)
    a.lib.bm_area_destroy(a.h)   # the library call alone, not the wrapper's cascade
    a.h = C.c_void_p()
    assert batch.lib.bm_batch_cycle(batch.h, 1) == F.BM_ERR_INVALID
    assert batch.lib.bm_batch_destroy(batch.h) == F.BM_OK
    batch.h = C.c_void_p()
    b.cycle(1)                   # the other area is unaffected
    b.close()
    ctx.close()
