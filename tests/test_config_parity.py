"""GPU parity at the benchmark workloads' own sizes, byte for byte against the
oracle (bismit's method restated in C and pinned to bismit's own kernels):

  * the 256 x 256 area (272,629,760 synapses), from its grown state and from
    a scrambled one, on both execution paths;
  * the 64 x 64 area for 1000 cycles from its grown state (strengths 0,
    learning on, seed 0), eagerly, in the plain form and as a graph-replayed
    batch of one, compared at checkpoints;
  * the 128 -> 192 -> 96 hierarchy with its tracts;
  * the 64 uneven instances as one autotuned, graph-replayed batch.

Scrambled states keep only SYN_PREV_ACTIVE in the synapse flags (the only
flag bit bismit writes), so the fused tuft kernel runs its specialised
consumers, as it does in the benchmarks; every test asserts the form each
fused tuft takes (bm_area_tuft_form) so the path under test is the one that
is measured. The stage semantics are cl/bismit.cl:695-747 (dendrites),
:755-842 (tufts), :888-915 (spiny stellate learning), :961-1022 (pyramidal
soma), :1195-1268 (distal learning) and cl/syns.cl:285-388 (synapses), in the
stage order of src/cortex/cortical_area.rs:716-789.
"""
import ctypes

import numpy as np
import pytest

import oracle
from bismit_b200 import _ffi as F, Cortex, configs, cortex, map as M
from helpers import diff_report, oracle_cortex_cycle, scramble

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = cortex._Ctx(0)
    yield c
    c.close()


def _forms(area):
    """{(layer, tuft): form} of every tuft of the area's data layers."""
    p = area.plan
    return {(i, t): area.tuft_form(i, t) for i in range(p.n_layers) for t in range(p.layers[i].n_tufts)}


def _strengths(plan, slab, layer):
    L = plan.layers[layer]
    off = int(L.buf_off[F.BUF["syn_strengths"]])
    return slab[off:off + int(L.n_syns)]


def _layer_of_kind(plan, kind):
    return next(i for i in range(plan.n_layers) if plan.layers[i].kind == kind)


def _check(plan, dev, ref, when):
    assert np.array_equal(dev, ref), "%s:\n%s" % (when, diff_report(plan, dev, ref))


@pytest.mark.parametrize("state", ["grown", "scrambled"])
@pytest.mark.parametrize("plain", [False, True], ids=["fused", "plain"])
def test_area_256_matches_oracle(ctx, state, plain):
    """The headline workload: 256 x 256 columns, spiny stellate 1 x 64,
    pyramidal depth 4 with proximal and distal 16 x 32 tufts, 3 % active
    frames, learning on. The fused path runs every tuft tiled with its
    specialised consumer (1 x 64 cells: shape 2; 16 x 32 cells: shape 6)."""
    lmaps, areas, act = configs.workload("area_256")
    st = configs.bench_settings()
    if plain:
        st.plain_kernels()
    area = cortex.CorticalArea(ctx, M.area_desc("v1", lmaps, areas, st), seed=1)
    plan = area.plan
    assert int(plan.n_syns_total) == 272629760
    slab = area.read_slab()
    if state == "scrambled":
        scramble(plan, slab, 11, clean_flags=True)
        area.write_slab(slab)
        area.set_cycle(0)
    forms = _forms(area)
    if plain:
        assert all(f["fused"] == 0 for f in forms.values())
    else:
        ssc = _layer_of_kind(plan, F.BM_LYR_SPINY_STELLATE)
        pyr = _layer_of_kind(plan, F.BM_LYR_PYRAMIDAL)
        for (i, t), f in forms.items():
            assert f["fused"] and f["tiled"] and f["footprint_tma"], (i, t, f)
            assert not f["flags_foreign"] and not f["sources_outside"], (i, t, f)
            assert f["consumer"] == (2 if i == ssc else 6), (i, t, f)
        assert forms[(pyr, 0)]["tile_w"] < plan.layers[pyr].u_size   # rows cut into parts
    # The spiny stellate tuft and inhibition run on the front stream, beside
    # the previous cycle's pyramidal steps (none on the plain path).
    assert area.front_steps() == (0 if plain else 2)
    n = 2 if plain else 3
    fr = configs.frames(n, area.input_len(), act, 5)
    ora = slab.copy()
    for k in range(n):
        area.write_input(fr[k])
        area.cycle(1)
        oracle.run(plan, ora, fr[k:k + 1], 1, start_cycle=k)
        _check(plan, area.read_slab(), ora, "cycle %d" % k)
    ssc = _layer_of_kind(plan, F.BM_LYR_SPINY_STELLATE)
    assert not np.array_equal(_strengths(plan, ora, ssc), _strengths(plan, slab, ssc))   # learning ran
    assert area.lib.bm_area_device_errors(area.h, ctypes.byref(ctypes.c_uint32())) == 0
    area.close()


@pytest.mark.parametrize("form", ["fused", "plain", "graph"])
def test_area_64_thousand_cycles(ctx, form):
    """The 64 x 64 configuration as stated: strengths start at 0, learning on,
    2 % active frames, seed 0, 1000 cycles; the whole slab is compared at
    cycles 1, 10, 100, 250, 500 and 1000. Frames come from device memory in
    one call per stretch; the graph form cycles the area as a batch of one
    replayed from a CUDA graph."""
    import torch
    lmaps, areas, act = configs.workload("area_64")
    st = configs.bench_settings()
    if form == "plain":
        st.plain_kernels()
    area = cortex.CorticalArea(ctx, M.area_desc("v1", lmaps, areas, st), seed=0)
    plan = area.plan
    flen = area.input_len()
    fr = configs.frames(1000, flen, act, 0)
    dev = torch.from_numpy(fr).to("cuda:0")
    torch.cuda.synchronize()
    batch = cortex.Batch(ctx, [area]) if form == "graph" else None
    if batch is not None:
        assert batch.frame_bytes() == flen
    if form != "plain":
        forms = _forms(area)
        ssc = _layer_of_kind(plan, F.BM_LYR_SPINY_STELLATE)
        assert forms[(ssc, 0)]["consumer"] == 1
        assert any(f["consumer"] == 6 for f in forms.values())   # the distal 16 x 32 tuft
    # Eager cycles from device frames overlap one cycle's spiny stellate chain
    # with the previous cycle's pyramidal steps (the front stream).
    assert area.front_steps() == (0 if form == "plain" else 2)
    ora = area.read_slab()
    start = ora.copy()
    done = 0
    for c in (1, 10, 100, 250, 500, 1000):
        n = c - done
        ptr = dev.data_ptr() + done * flen
        if batch is not None:
            batch.cycle_frames_device(ptr, n)
        else:
            area.cycle_frames_device(ptr, flen, n)
        oracle.run(plan, ora, fr[done:c], n, start_cycle=done)
        _check(plan, area.read_slab(), ora, "cycle %d" % c)
        done = c
    assert area.cycle_count() == 1000
    pyr = _layer_of_kind(plan, F.BM_LYR_PYRAMIDAL)
    for i in (_layer_of_kind(plan, F.BM_LYR_SPINY_STELLATE), pyr):
        assert not np.array_equal(_strengths(plan, ora, i), _strengths(plan, start, i)), i
    if batch is not None:
        assert batch.device_errors() == 0
        batch.close()
    area.close()


def test_hierarchy_full_size_matches_oracle(ctx):
    """The three-area hierarchy at its configured sizes (128 -> 192 -> 96,
    pyramidal depth 2, two feed-forward and two feedback tracts), batched and
    graph-replayed, from scrambled states, 3 cycles."""
    lm, ar, names = configs.hierarchy()
    cx = Cortex.builder(lm, ar).ca_settings(configs.bench_settings()).seed(3).build()
    plans = [cx.area(n).plan for n in names]
    assert [int(p.v_size) for p in plans] == [128, 192, 96]
    assert len(cx.tracts) == 4
    slabs = []
    for k, n in enumerate(names):
        s = cx.area(n).read_slab()
        scramble(plans[k], s, 40 + k, clean_flags=True)
        cx.area(n).write_slab(s)
        cx.area(n).set_cycle(0)
        slabs.append(s.copy())
        assert any(f["consumer"] for f in _forms(cx.area(n)).values())
    fr = configs.frames(3, 128 * 128, 0.02, 5)
    v1 = cx.area("v1")
    for c in range(3):
        v1.write_input(fr[c])
        cx.cycle()
        oracle_cortex_cycle(plans, slabs, cx.tracts, fr[c], c)
        for k, n in enumerate(names):
            _check(plans[k], cx.area(n).read_slab(), slabs[k], "cycle %d, %s" % (c, n))
    cx.close()


def test_batch_64_instances_match_oracle(ctx):
    """The 64 uneven instances (sides 32..192, depth 1..4, distal {8,16} x
    {16,32,64}, 1-4 % active), autotuned as the benchmark does, cycled as one
    graph-replayed batch from scrambled states: every instance equals the
    oracle after each of 2 cycles."""
    import torch
    ins = configs.batch_instances(64, 0)
    areas, frames, slabs = [], [], []
    for i, (side, depth, dens, syns, act) in enumerate(ins):
        lmaps, ar = configs.instance_area(side, depth, dens, syns)
        a = cortex.CorticalArea(ctx, M.area_desc("v1", lmaps, ar, configs.bench_settings()), 1000 + i)
        s = a.read_slab()
        scramble(a.plan, s, 500 + i, clean_flags=True)
        a.write_slab(s)
        a.set_cycle(0)
        areas.append(a)
        slabs.append(s)
        frames.append(configs.frames(2, a.input_len(), act, 1000 + i))
    assert sum(int(a.plan.n_syns_total) for a in areas) == 1120346368
    batch = cortex.Batch(ctx, areas)
    batch.autotune(None)   # trial cycles restore the state they touch
    for k, a in enumerate(areas):
        _check(a.plan, a.read_slab(), slabs[k], "area %d after autotuning" % k)
    shapes = set()
    for a in areas:
        shapes |= {f["consumer"] for f in _forms(a).values() if f["fused"]}
    assert {1, 3, 4, 5, 6, 7, 8} <= shapes, shapes   # every specialised consumer the sizes reach
    packed = torch.from_numpy(batch.pack_frames(frames)).to("cuda:0")
    fb = batch.frame_bytes()
    torch.cuda.synchronize()
    for c in range(2):
        batch.cycle_frames_device(packed.data_ptr() + c * fb, 1)
        for k, a in enumerate(areas):
            oracle.run(a.plan, slabs[k], frames[k][c:c + 1], 1, start_cycle=c)
            _check(a.plan, a.read_slab(), slabs[k], "cycle %d, instance %d %s" % (c, k, ins[k][:4]))
    assert batch.device_errors() == 0
    batch.close()
    for a in areas:
        a.close()
