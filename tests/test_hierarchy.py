"""Multi-area cortex: the hierarchy v1 -> v2 -> v3 with feed-forward and
feedback tracts, batched, against the oracle run area by area with the same
tract timing (every tract carries its source's output of the previous cycle).
"""
import numpy as np
import pytest

from bismit_b200 import Cortex, configs, map as M, plan_of
from helpers import diff_report, oracle_cortex_cycle, oracle_cortex_cycle_in_order, scramble

SIDES = (32, 48, 24)


def test_tract_routing_of_the_hierarchy():
    lm, ar, names = configs.hierarchy(SIDES)
    plans = [plan_of(M.area_desc(n, lm, ar, configs.bench_settings()), 1) for n in names]
    tracts, external = M.area_tracts(lm, ar, names, plans)
    # v2.iii -> v1.eff_in, v1.iii -> v2.aff_in, v3.iii -> v2.eff_in, v2.iii -> v3.aff_in
    assert sorted((s, d, i) for (s, _o, d, i, _off, _n) in tracts) == [(0, 1, 0), (1, 0, 1), (1, 2, 0), (2, 1, 1)]
    for (s, o, d, i, off, n) in tracts:
        assert n == int(plans[s].outputs[o].len) and off + n <= int(plans[d].inputs[i].len)
    assert external == [(0, 0, 0, SIDES[0] ** 2, "v0", "ganglion")]


def _with_filters(lm, ar):
    """Retina chains on an external input (v1), on a tract-fed feed-forward
    input two slices deep (v2, two filters) and on a feedback input (v2)."""
    ar.by_name("v1").filter_chain(M.InputTrack.Afferent, [M.THAL_SP], ["retina"])
    ar.by_name("v2").filter_chain(M.InputTrack.Afferent, [M.THAL_SP], ["retina", "retina"])
    ar.by_name("v2").filter_chain(M.InputTrack.Efferent, [M.THAL_SP], ["retina"])
    return lm, ar


@pytest.mark.gpu
@pytest.mark.parametrize("filters", [False, True], ids=["plain_inputs", "filtered_inputs"])
def test_hierarchy_matches_oracle(filters):
    lm, ar, names = configs.hierarchy(SIDES)
    if filters:
        _with_filters(lm, ar)
    cx = Cortex.builder(lm, ar).ca_settings(configs.bench_settings()).seed(3).build()
    plans = [cx.area(n).plan for n in names]
    assert sum(int(p.n_filter_chains) for p in plans) == (3 if filters else 0)
    slabs = []
    for k, n in enumerate(names):
        s = cx.area(n).read_slab()
        scramble(plans[k], s, 40 + k)
        cx.area(n).write_slab(s)
        cx.area(n).set_cycle(0)
        slabs.append(s.copy())
    fr = configs.frames(6, SIDES[0] ** 2, 0.02, 5)
    v1 = cx.area("v1")
    for c in range(6):
        v1.write_input(fr[c])
        cx.cycle()
        oracle_cortex_cycle(plans, slabs, cx.tracts, fr[c], c)
        for k, n in enumerate(names):
            dev = cx.area(n).read_slab()
            assert np.array_equal(dev, slabs[k]), "cycle %d, %s:\n%s" % (c, n, diff_report(plans[k], dev, slabs[k]))
    cx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("filters", [False, True], ids=["plain_inputs", "filtered_inputs"])
def test_same_cycle_tracts_match_oracle(filters):
    """bismit's own tract timing (Cortex::cycle cycles the areas in order,
    src/cortex/cortex.rs:99-119): a feed-forward tract carries its source's
    output of the same cycle, a feedback tract the previous cycle's; against
    the oracle cycling the areas in the same order."""
    from bismit_b200.cortex import SAME_CYCLE
    lm, ar, names = configs.hierarchy(SIDES)
    if filters:
        _with_filters(lm, ar)
    cx = Cortex.builder(lm, ar).ca_settings(configs.bench_settings()).seed(3).tract_timing(SAME_CYCLE).build()
    assert cx.batch is None
    plans = [cx.area(n).plan for n in names]
    slabs = []
    for k, n in enumerate(names):
        s = cx.area(n).read_slab()
        scramble(plans[k], s, 60 + k, clean_flags=True)
        cx.area(n).write_slab(s)
        cx.area(n).set_cycle(0)
        slabs.append(s.copy())
    fr = configs.frames(5, SIDES[0] ** 2, 0.02, 7)
    v1 = cx.area("v1")
    for c in range(5):
        v1.write_input(fr[c])
        cx.cycle()
        oracle_cortex_cycle_in_order(plans, slabs, cx.tracts, fr[c], c)
        for k, n in enumerate(names):
            dev = cx.area(n).read_slab()
            assert np.array_equal(dev, slabs[k]), "cycle %d, %s:\n%s" % (c, n, diff_report(plans[k], dev, slabs[k]))
    cx.close()


def test_same_cycle_timing_differs_from_previous_cycle():
    """The two timings are different methods: on the oracle, the hierarchy's
    second area ends a few cycles in a different state under each (so the
    same-cycle test above could not pass by accident)."""
    import oracle
    from bismit_b200 import plan_of
    lm, ar, names = configs.hierarchy(SIDES)
    plans = [plan_of(M.area_desc(n, lm, ar, configs.bench_settings()), 1) for n in names]
    tracts, _ext = M.area_tracts(lm, ar, names, plans)
    base = []
    for k, p in enumerate(plans):
        s = np.zeros(int(p.slab_bytes), np.uint8)
        oracle.grow(p, s, 1, 0)
        scramble(p, s, 70 + k, clean_flags=True)
        base.append(s)
    a = [s.copy() for s in base]
    b = [s.copy() for s in base]
    fr = configs.frames(4, SIDES[0] ** 2, 0.05, 8)
    for c in range(4):
        oracle_cortex_cycle(plans, a, tracts, fr[c], c)
        oracle_cortex_cycle_in_order(plans, b, tracts, fr[c], c)
    assert not np.array_equal(a[1], b[1])


@pytest.mark.gpu
@pytest.mark.parametrize("delivery", ["api", "raw"])
def test_unbatched_tracts_without_reads_match_oracle(delivery):
    """Areas cycled one after another with every tract delivered at the head
    of each cycle (the batched path's timing), six cycles queued with no read
    in between, so that each area's front steps could run ahead of a tract's
    copy: through bm_area_deliver_tract ("api"), or by the caller's own copies
    on the area's stream followed by bm_area_axons_touched ("raw")."""
    import torch
    from bismit_b200.cortex import SAME_CYCLE
    lm, ar, names = configs.hierarchy(SIDES)
    cx = Cortex.builder(lm, ar).ca_settings(configs.bench_settings()).seed(5).tract_timing(SAME_CYCLE).build()
    stream = torch.cuda.Stream()
    cx.ctx.set_stream(stream.cuda_stream)
    areas = [cx.area(n) for n in names]
    plans = [a.plan for a in areas]
    assert any(a.front_steps() for a in areas)
    slabs = []
    for k, a in enumerate(areas):
        s = a.read_slab()
        scramble(plans[k], s, 80 + k, clean_flags=True)
        a.write_slab(s)
        a.set_cycle(0)
        slabs.append(s.copy())
    copies = []
    for (sk, so, dk, di, off, n) in cx.tracts:
        ps, pd = plans[sk], plans[dk]
        src = areas[sk].slab_ptr() + int(ps.axon_off) + int(ps.outputs[so].axn_idz)
        dst = areas[dk].slab_ptr() + int(pd.axon_off) + int(pd.inputs[di].axn_idz) + int(off)
        copies.append((_dev_bytes(src, n), _dev_bytes(dst, n)))
    fr = configs.frames(6, SIDES[0] ** 2, 0.03, 9)
    with torch.cuda.stream(stream):
        for c in range(6):
            if delivery == "api":
                for (sk, so, dk, di, off, _n) in cx.tracts:
                    areas[dk].deliver_tract(areas[sk], so, di, off)
            else:
                for src, dst in copies:
                    dst.copy_(src)
                for a in areas:   # every area's axons were read or written
                    a.axons_touched()
            areas[0].write_input(fr[c])
            for a in areas:
                a.cycle(1)
    for c in range(6):
        oracle_cortex_cycle(plans, slabs, cx.tracts, fr[c], c)
    for k, n in enumerate(names):
        dev = areas[k].read_slab()
        assert np.array_equal(dev, slabs[k]), "%s:\n%s" % (n, diff_report(plans[k], dev, slabs[k]))
    cx.close()


def _dev_bytes(ptr, n):
    """A torch u8 tensor over n bytes of device memory at ptr."""
    import torch

    class _View:
        __cuda_array_interface__ = {"shape": (int(n),), "typestr": "|u1", "data": (int(ptr), False),
                                    "version": 3, "strides": None, "stream": None}
    return torch.as_tensor(_View(), device="cuda")
