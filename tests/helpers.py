"""Shared test helpers: schemes, seeded initial states, buffer diffs, digests."""
import hashlib

import numpy as np

from bismit_b200 import _ffi as F, configs, map as M, plan_of

NO_BUF = 2 ** 64 - 1

SCHEMES = {
    "testbed": lambda: configs.testbed_area(),
    "mixed": lambda: configs.mixed_area(),
    "area_64": lambda: configs.workload("area_64")[:2],
    "area_48_deep": lambda: configs.workload("area_48_deep")[:2],
    "smoother": lambda: configs.smoother_area(),
    "testbed_retina": lambda: configs.testbed_area(retina=True),
    "retina": lambda: configs.retina_area(48, n_filters=2, src_depth=2),
    "retina_scaled": lambda: configs.retina_area(64, n_filters=3, src_side=32),
    # The 256 x 256 workload's layer shapes on a 48 x 48 grid: spiny stellate
    # 1 x 64, pyramidal depth 4 with proximal and distal 16 x 32 tufts at
    # reach 6 (the specialised consumers of both layer kinds, in seconds).
    "area_256_shape": lambda: configs.workload("area_256_shape")[:2],
    # A batched instance's largest cells: pyramidal depth 2 with a distal
    # 16 x 64 tuft (1024 synapses a cell, one warp's unit in two halves).
    "distal_1024": lambda: configs.instance_area(48, 2, 16, 64),
}


def settings_for(kind="default", plain=False):
    """Regrowth is off except for kind "regrowth" (the reference's parity runs
    set disable_regrowth)."""
    s = M.CorticalAreaSettings()
    if kind != "regrowth":
        s.disable_regrowth()
    if kind == "bypass_inhib":
        s.bypass_inhib()
    elif kind == "no_learning":
        s.disable_learning()
    elif kind == "no_pyrs":
        s.disable_pyrs()
    elif kind == "no_sscs":
        s.disable_sscs()
    elif kind == "bypass_filters":
        s.bypass_filters()
    elif kind == "zero_strength":
        s.strengths_start_at_zero()
    if plain:
        s.plain_kernels()
    return s


def desc_of(scheme, settings=None):
    lmaps, areas = SCHEMES[scheme]()
    return M.area_desc("v1", lmaps, areas, settings or settings_for())


def plan_for(scheme, settings=None, seed=7):
    d = desc_of(scheme, settings)
    return d, plan_of(d, seed)


def buffers(plan):
    """(label, offset, length) of every buffer in the slab."""
    out = [("axon_states", int(plan.axon_off), int(plan.n_axons))]
    for l in range(plan.n_layers):
        L = plan.layers[l]
        for k, n in enumerate(F.BUF_NAMES):
            if L.buf_off[k] != NO_BUF:
                out.append(("L%d.%s" % (l, n), int(L.buf_off[k]), int(L.buf_len[k])))
    for c in range(plan.n_filter_chains):
        ch = plan.filter_chains[c]
        for k in range(ch.n_filters):
            out.append(("filter%d.in%d" % (c, k), int(ch.buf_off[k]), int(ch.depth * ch.v_size * ch.u_size)))
    return out


def named(plan, slab):
    """{label: bytes} of every buffer of the slab."""
    return {name: slab[off:off + n] for name, off, n in buffers(plan)}


def diff_report(plan, a, b, limit=12):
    lines = []
    for name, off, n in buffers(plan):
        x, y = a[off:off + n], b[off:off + n]
        if not np.array_equal(x, y):
            idx = np.nonzero(x != y)[0]
            lines.append("%s: %d of %d differ (first %d: %s vs %s)" % (
                name, idx.size, n, idx[0], x[idx[:4]].tolist(), y[idx[:4]].tolist()))
    return "\n".join(lines[:limit])


def digests(plan, slab):
    return {name: hashlib.sha256(slab[off:off + n].tobytes()).hexdigest()[:32] for name, off, n in buffers(plan)}


def scramble(plan, slab, seed, clean_flags=False):
    """Overwrites the cycle state (not the synapse sources) with seeded values so
    every branch of the kernels is reached: energies at and above the restless
    and dark cutoffs, flags with unrelated bits set, strengths over the whole i8
    range (including -128 and 127), prior synapse and tuft states.

    With clean_flags the synapse flags keep only SYN_PREV_ACTIVE (0x10), the
    only bit bismit's kernels ever write (cl/syns.cl:23-33): the state real
    runs are in, which the fused kernel serves with its specialised consumers
    (foreign bits send it to the form that streams flags through)."""
    rng = np.random.default_rng([seed, 0x5C7A])
    for l in range(plan.n_layers):
        L = plan.layers[l]

        def put(k, vals):
            off = int(L.buf_off[k])
            slab[off:off + len(vals)] = vals

        n_syn, n_den, n_cel = int(L.n_syns), int(L.n_dens), int(L.cells)
        st = rng.integers(0, 256, n_syn, dtype=np.uint8)
        st[rng.random(n_syn) < 0.7] = 0
        put(F.BUF["syn_states"], st)
        put(F.BUF["syn_strengths"], rng.integers(-128, 128, n_syn).astype(np.int8).view(np.uint8))
        put(F.BUF["syn_flag_sets"], rng.integers(0, 256, n_syn, dtype=np.uint8))
        for k in ("den_activities", "den_energies", "den_states", "den_states_raw"):
            put(F.BUF[k], rng.integers(0, 256, n_den, dtype=np.uint8))
        en = rng.integers(0, 256, n_cel, dtype=np.uint8)
        en[rng.random(n_cel) < 0.05] = 255
        put(F.BUF["cel_energies"], en)
        put(F.BUF["cel_activities"], rng.integers(0, 256, n_cel, dtype=np.uint8))
        if L.kind == F.BM_LYR_PYRAMIDAL:
            n_ct = int(L.n_celtfts)
            for k in ("tft_prev_best_den_ids", "tft_best_den_ids"):
                put(F.BUF[k], np.concatenate([rng.integers(0, int(L.tufts[t].dens_per_tft), n_cel, dtype=np.uint8)
                                              for t in range(L.n_tufts)]))
            for k in ("tft_prev_best_den_states_raw", "tft_prev_best_den_states", "tft_prev_states",
                      "tft_best_den_states_raw", "tft_best_den_states", "tft_states"):
                v = rng.integers(0, 256, n_ct, dtype=np.uint8)
                v[rng.random(n_ct) < 0.3] = 0
                put(F.BUF[k], v)
            put(F.BUF["cel_flag_sets"], rng.integers(0, 256, n_cel, dtype=np.uint8))
            put(F.BUF["cel_states"], rng.integers(0, 256, n_cel, dtype=np.uint8))
    ax = rng.integers(0, 256, int(plan.n_axons), dtype=np.uint8)
    ax[rng.random(int(plan.n_axons)) < 0.8] = 0
    slab[int(plan.axon_off):int(plan.axon_off) + int(plan.n_axons)] = ax
    if clean_flags:
        for l in range(plan.n_layers):
            L = plan.layers[l]
            off = int(L.buf_off[F.BUF["syn_flag_sets"]])
            slab[off:off + int(L.n_syns)] &= 0x10


def initial_slab(plan, grow_seed, scramble_seed=None, init_flags=0, clean_flags=False):
    import oracle
    slab = np.zeros(int(plan.slab_bytes), np.uint8)
    oracle.grow(plan, slab, grow_seed, init_flags)
    if scramble_seed is not None:
        scramble(plan, slab, scramble_seed, clean_flags=clean_flags)
    return slab


def frames_for(plan, n, seed, active=0.05):
    if plan.n_inputs == 0:
        return None
    return configs.frames(n, int(plan.inputs[0].len), active, seed)


def oracle_cortex_cycle(plans, slabs, tracts, ext_frame, cycle):
    """One cycle of a multi-area cortex on the oracle with the batched path's
    tract timing: every tract first delivers its source's output of the
    previous cycle, the external frame goes into area 0's first input, then
    each area cycles."""
    import oracle
    outs = [s[int(p.axon_off):].copy() for p, s in zip(plans, slabs)]
    for (s, o, d, i, off, n) in tracts:
        src = int(plans[s].outputs[o].axn_idz)
        oracle.intake(plans[d], slabs[d], i, off, outs[s][src:src + n])
    oracle.intake(plans[0], slabs[0], 0, 0, ext_frame)
    for p, s in zip(plans, slabs):
        oracle.run(p, s, None, 1, start_cycle=cycle)


def oracle_cortex_cycle_in_order(plans, slabs, tracts, ext_frame, cycle):
    """One cycle of a multi-area cortex on the oracle in bismit's own order
    (Cortex::cycle, src/cortex/cortex.rs:99-119): area after area, each
    taking its tracts' current outputs -- an earlier area's of this cycle, a
    later area's of the previous one -- and area 0 its external frame, then
    cycling."""
    import oracle
    for k, (p, s) in enumerate(zip(plans, slabs)):
        for (sk, o, d, i, off, n) in tracts:
            if d != k:
                continue
            src = int(plans[sk].axon_off) + int(plans[sk].outputs[o].axn_idz)
            oracle.intake(p, s, i, off, slabs[sk][src:src + n].copy())
        if k == 0:
            oracle.intake(p, s, 0, 0, ext_frame)
        oracle.run(p, s, None, 1, start_cycle=cycle)
