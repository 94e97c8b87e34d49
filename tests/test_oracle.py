"""CPU: the C restatement oracle pinned against bismit's own OpenCL kernels
(cl/bismit.cl, cl/syns.cl, cl/control.cl compiled for the CPU by oracle/ref),
plus the reference's own known-answer tests for this path."""
import ctypes

import numpy as np
import pytest

import oracle
from bismit_b200 import _ffi as F, configs, map as M
from helpers import diff_report, frames_for, initial_slab, plan_for, scramble, settings_for


@pytest.mark.parametrize("scheme", ["testbed", "mixed", "area_64", "area_48_deep", "smoother", "testbed_retina",
                                    "retina", "retina_scaled"])
@pytest.mark.parametrize("kind", ["default", "bypass_inhib", "no_learning", "zero_strength"])
def test_port_matches_reference_kernels(ref_oracle, scheme, kind):
    _, plan = plan_for(scheme, settings_for(kind))
    slab = initial_slab(plan, 7, scramble_seed=11)
    fr = frames_for(plan, 8, 5)
    a, b = slab.copy(), slab.copy()
    for k in range(8):
        f = None if fr is None else fr[k:k + 1]
        oracle.run(plan, a, f, 1, start_cycle=k, impl="port")
        oracle.run(plan, b, f, 1, start_cycle=k, impl="ref")
        assert np.array_equal(a, b), "cycle %d:\n%s" % (k, diff_report(plan, a, b))


def test_port_matches_reference_kernels_long(ref_oracle):
    """80 cycles from the grown state: learning accumulates in both."""
    _, plan = plan_for("area_64", settings_for("zero_strength"))
    slab = initial_slab(plan, 3, init_flags=F.BM_INIT_STRENGTH_ZERO)
    fr = frames_for(plan, 80, 2, active=0.02)
    a, b = slab.copy(), slab.copy()
    oracle.run(plan, a, fr, 80, impl="port")
    oracle.run(plan, b, fr, 80, impl="ref")
    assert np.array_equal(a, b), diff_report(plan, a, b)
    L0 = plan.layers[0]
    s = a[L0.buf_off[F.BUF["syn_strengths"]]:][:L0.n_syns].view(np.int8)
    assert (s != 0).mean() > 0.01, "spiny stellate learning changed no strength"


def test_axon_index_scalar_equals_vec4(ref_oracle):
    """src/tests/kernels.rs:21-91: test_axn_idxs_scl and test_axn_idxs_vec4 give
    identical axon indices for shuffled offsets in +-SYNAPSE_REACH (8)."""
    _, plan = plan_for("testbed")
    rng = np.random.default_rng(0)
    depth, v, u = int(plan.n_slices), 24, 24
    n = depth * v * u
    vo = rng.permutation(np.resize(np.arange(-8, 9, dtype=np.int8), n))
    uo = rng.permutation(np.resize(np.arange(-8, 9, dtype=np.int8), n))
    scl, vec = oracle.ref_axn_idxs(plan, depth, v, u, vo, uo)
    assert np.array_equal(scl, vec)
    # The restatement gives the same indices.
    port = oracle.load_port()
    safe = ctypes.c_int()
    got = np.zeros(n, np.uint32)
    for i in range(n):
        s, vv, uu = i // (v * u), (i // u) % v, i % u
        got[i] = port.bmo_axn_idx_scl(ctypes.byref(plan), s, vv, int(vo[i]), uu, int(uo[i]), ctypes.byref(safe))
    assert np.array_equal(got, scl)


@pytest.mark.parametrize("r", [0, 1, 2, 3, 4, 6, 8, 16])
def test_hex_offsets_count_and_symmetry(r):
    """gen_syn_offs (src/map/syn_src.rs:47-149) at scale 16 is the hex disk of
    radius r: 3r(r+1)+1 tiles, symmetric, max(|v|,|u|,|v+u|) <= r."""
    v, u = oracle.gen_syn_offs(r, 16, 16)
    assert len(v) == 3 * r * (r + 1) + 1
    pts = set(zip(v.tolist(), u.tolist()))
    assert len(pts) == len(v)
    assert all(max(abs(a), abs(b), abs(a + b)) <= r for a, b in pts)
    assert all((-a, -b) in pts for a, b in pts)


def test_rnd_stream_is_deterministic_and_keyed():
    a = [oracle.rnd(5, 1, 2, F.BM_RND_DEN_CYCLE, 0, c) for c in range(100)]
    b = [oracle.rnd(5, 1, 2, F.BM_RND_DEN_CYCLE, 0, c) for c in range(100)]
    assert a == b
    assert len(set(a)) == 100
    assert oracle.rnd(5, 1, 2, F.BM_RND_DEN_CYCLE, 1, 0) != a[0]
    assert oracle.rnd(6, 1, 2, F.BM_RND_DEN_CYCLE, 0, 0) != a[0]
    lib = F.lib()
    assert [lib.bm_rnd(5, 1, 2, F.BM_RND_DEN_CYCLE, 0, c) for c in range(100)] == a


def test_smoother_only_nudges_energies():
    """One cycle with and without the activity smoothers from the same state:
    only the hosts' cell energies differ, each by at most one step per lattice
    (six), and some do (src/cortex/smoother.rs, cl/control.cl:227-295)."""
    from bismit_b200 import plan_of
    from helpers import named
    with_s = M.area_desc("v1", *configs.smoother_area(), configs.bench_settings())
    without = M.area_desc("v1", *configs.smoother_area(smoothers=False), configs.bench_settings())
    p1, p0 = plan_of(with_s, 7), plan_of(without, 7)
    a = np.zeros(int(p1.slab_bytes), np.uint8)
    oracle.grow(p1, a, 7, 0)
    scramble(p1, a, 11)
    b = a.copy()
    assert p0.slab_bytes == p1.slab_bytes
    fr = configs.frames(1, int(p1.inputs[0].len), 0.05, 5)
    oracle.run(p1, a, fr, 1, start_cycle=0)
    oracle.run(p0, b, fr, 1, start_cycle=0)
    na, nb = named(p1, a), named(p0, b)
    moved = 0
    for name in nb:
        if name.endswith("cel_energies"):
            d = na[name].astype(int) - nb[name].astype(int)
            assert np.abs(d).max() <= 6
            moved += int(np.count_nonzero(d))
        else:
            assert np.array_equal(na[name], nb[name]), name
    assert moved > 0


def _retina_py(grid):
    """retina (cl/filters.cl:34-100) over a (depth, v, u) uint8 grid, written
    out loop by loop from the kernel text: the cell index picks off-center
    (bit 0) and large (bit 1 xor bit 0) cells, the hexagon of radius 5 or 3
    is averaged with cells outside the grid read as 0, and the cell's output
    is its margin over the threshold 48 (cl/bismit.cl:19)."""
    depth, vs, us = grid.shape
    out = np.zeros_like(grid)
    for s in range(depth):
        for v in range(vs):
            for u in range(us):
                i = (s * vs + v) * us + u
                off_cen = i & 1
                large = ((i & 3) >> 1) ^ off_cen
                r = 5 if large else 3
                tot = cnt = 0
                for vo in range(-r, r + 1):
                    for uo in range(max(-r, -vo - r), min(r, -vo + r) + 1):
                        vv, uu = v + vo, u + uo
                        if 0 <= vv < vs and 0 <= uu < us:
                            tot += int(grid[s, vv, uu])
                        cnt += 1
                avg, c = tot // cnt, int(grid[s, v, u])
                if off_cen:
                    out[s, v, u] = avg - (c + 48) if avg > c + 48 else 0
                else:
                    out[s, v, u] = c - (avg + 48) if c > avg + 48 else 0
    return out


@pytest.mark.parametrize("n_filters,depth", [(1, 1), (1, 2), (2, 2)])
def test_retina_filter_known_answers(n_filters, depth):
    """The input axons after a cycle are the retina chain applied to the frame
    (each filter of a chain of two reads the previous one's whole output, the
    slices of a two-deep source being back to back from axon 0); bypassing the
    filters leaves the frame itself; a cycle without a new frame filters the
    same stored frame again, not the filtered output."""
    from bismit_b200 import plan_of
    side = 16
    for bypass in (False, True):
        st = configs.bench_settings()
        if bypass:
            st.bypass_filters()
        plan = plan_of(M.area_desc("v1", *configs.retina_area(side, n_filters, depth), st), 3)
        assert plan.n_filter_chains == 1
        io = plan.inputs[0]
        assert io.len == depth * side * side
        slab = np.zeros(int(plan.slab_bytes), np.uint8)
        oracle.grow(plan, slab, 3, 0)
        rng = np.random.default_rng(depth * 10 + n_filters)
        frame = rng.integers(0, 256, size=(1, io.len), dtype=np.uint8)
        frame[0, rng.random(io.len) < 0.5] = 0     # sparse enough for both cell kinds to fire
        want = frame[0].reshape(depth, side, side)
        if not bypass:
            for _ in range(n_filters):
                want = _retina_py(want)
            assert np.count_nonzero(want) > 0
        a0 = int(plan.axon_off + io.axn_idz)
        oracle.run(plan, slab, frame, 1, start_cycle=0)
        assert np.array_equal(slab[a0:a0 + io.len], want.reshape(-1))
        oracle.run(plan, slab, None, 1, start_cycle=1)
        assert np.array_equal(slab[a0:a0 + io.len], want.reshape(-1))


def test_filter_chain_plans_and_refusals():
    """Chains resolve to the source their signature names, with one
    depth x v x u buffer per filter; source dims that are not multiples of 8
    (the 1 x 8 x 8 work-groups of SensoryFilter::new) and unknown or custom
    filters are refused."""
    from bismit_b200 import plan_of
    plan = plan_of(M.area_desc("v1", *configs.retina_area(64, 3, 1, src_side=32), configs.bench_settings()), 1)
    c = plan.filter_chains[0]
    assert (c.input, c.frame_off, c.tar_slc, c.depth, c.v_size, c.u_size, c.n_filters) == (0, 0, 0, 1, 32, 32, 3)
    assert all(c.filters[k] == F.BM_FILTER_RETINA for k in range(3))
    offs = [int(c.buf_off[k]) for k in range(3)]
    assert all(o % 256 == 0 for o in offs) and offs == sorted(offs) and offs[-1] + 1024 <= plan.slab_bytes
    with pytest.raises(F.BismitError, match="multiples of 8"):
        plan_of(M.area_desc("v1", *configs.retina_area(44), configs.bench_settings()), 1)
    with pytest.raises(ValueError, match="unknown filter"):
        M.FilterScheme("sharpen")
    with pytest.raises(ValueError, match="custom OpenCL"):
        M.FilterScheme("retina", "my_filters.cl")
    lmaps, areas = configs.retina_area(48)
    areas.by_name("v1").filter_chain(M.InputTrack.Efferent, [M.THAL_SP], ["retina"])
    with pytest.raises(ValueError, match="Unable to find a layer"):
        M.area_desc("v1", lmaps, areas, configs.bench_settings())


def _plan_cases():
    """Every area scheme the tests and benchmarks use, as (label, desc)."""
    from helpers import SCHEMES
    out = []
    for name in sorted(SCHEMES):
        lm, ar = SCHEMES[name]()
        for kind in ("default", "regrowth"):
            out.append(("%s/%s" % (name, kind), M.area_desc("v1", lm, ar, settings_for(kind))))
    for w in ("area_64", "area_256"):
        lm, ar, _ = configs.workload(w)
        out.append((w, M.area_desc("v1", lm, ar, configs.bench_settings())))
    for i, (side, depth, dens, syns, _a) in enumerate(configs.batch_instances(64, 0)[:12]):
        lm, ar = configs.instance_area(side, depth, dens, syns)
        out.append(("instance%d" % i, M.area_desc("v1", lm, ar, configs.bench_settings())))
    lm, ar, names = configs.hierarchy()
    for n in names:
        out.append(("hierarchy/" + n, M.area_desc(n, lm, ar, configs.bench_settings())))
    return out


def test_oracle_plan_resolver_agrees_with_the_library():
    """The oracle's own restatement of bismit's slice map and index spaces
    (oracle/plan.py) and the library's bm_plan_resolve give the same plan,
    byte for byte, for every scheme in use; so the oracle and the CPU
    reference arm stand on a plan the library did not make."""
    from bismit_b200 import plan_of
    from oracle import plan as OP
    for label, d in _plan_cases():
        mine = OP.resolve(d, 7)
        lib = plan_of(d, 7)
        a, b = bytes(mine), bytes(lib)
        assert a == b, "%s: plans differ at byte %d" % (label, next(i for i in range(len(a)) if a[i] != b[i]))


def test_oracle_plan_resolver_refuses_what_the_library_refuses():
    from bismit_b200 import plan_of
    from oracle import plan as OP
    lm, ar, _ = configs.workload("area_64")
    bad = []
    d = M.area_desc("v1", lm, ar, configs.bench_settings())
    d.layers[3].tufts[0].dens_per_tft = 0
    bad.append(d)
    d = M.area_desc("v1", lm, ar, configs.bench_settings())
    d.layers[3].tufts[1].syns_per_den = 4096   # more than the pool's offsets
    bad.append(d)
    d = M.area_desc("v1", lm, ar, configs.bench_settings())
    d.layers[3].tufts[1].src[0].prevalence = 0
    bad.append(d)
    for d in bad:
        with pytest.raises(OP.PlanError):
            OP.resolve(d, 0)
        with pytest.raises(F.BismitError):
            plan_of(d, 0)
