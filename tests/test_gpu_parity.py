"""GPU parity: the CUDA path against the CPU oracle, byte for byte.

Every test drives the device through the C ABI (bismit_b200.cortex wraps
include/bismit_b200.h) and compares the whole state slab (every axon,
synapse, dendrite, tuft and cell buffer) with the oracle after every cycle,
so a divergence is reported at the cycle and buffer where it first appears.
"""
import numpy as np
import pytest

import oracle
from bismit_b200 import _ffi as F, cortex
from helpers import buffers, desc_of, diff_report, frames_for, initial_slab, settings_for

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = cortex._Ctx(0)
    yield c
    c.close()


def _area(ctx, scheme, settings, seed=7):
    return cortex.CorticalArea(ctx, desc_of(scheme, settings), seed)


@pytest.mark.parametrize("scheme", ["testbed", "mixed", "area_64", "area_48_deep"])
@pytest.mark.parametrize("flags", [0, F.BM_INIT_STRENGTH_ZERO])
def test_growth_matches_oracle(ctx, scheme, flags):
    s = settings_for()
    s.init_flags = flags
    area = _area(ctx, scheme, s, seed=123)
    dev = area.read_slab()
    ref = np.zeros(area.slab_bytes, np.uint8)
    oracle.grow(area.plan, ref, 123, flags)
    assert np.array_equal(dev, ref), diff_report(area.plan, dev, ref)
    area.close()


def _run_parity(ctx, scheme, kind, plain, cycles, scramble=True, active=0.05, start=0, clean_flags=False,
                consumers=None, footprint_tma=None):
    s = settings_for(kind, plain=plain)
    area = _area(ctx, scheme, s)
    plan = area.plan
    slab = initial_slab(plan, 7, scramble_seed=11 if scramble else None, clean_flags=clean_flags)
    area.write_slab(slab)
    area.set_cycle(start)
    if consumers is not None:
        forms = [area.tuft_form(i, t) for i in range(plan.n_layers) for t in range(plan.layers[i].n_tufts)]
        got = {f["consumer"] for f in forms}
        assert set(consumers) <= got, got
        if footprint_tma is not None:
            assert any(f["footprint_tma"] for f in forms) == footprint_tma, forms
    fr = frames_for(plan, cycles, 5, active)
    ora = slab.copy()
    for k in range(cycles):
        if fr is not None:
            area.write_input(fr[k])
        area.cycle(1)
        oracle.run(plan, ora, None if fr is None else fr[k:k + 1], 1, start_cycle=start + k)
        dev = area.read_slab()
        assert np.array_equal(dev, ora), "cycle %d:\n%s" % (start + k, diff_report(plan, dev, ora))
    area.close()
    return plan, slab, ora


@pytest.mark.parametrize("plain", [True, False], ids=["plain", "fused"])
@pytest.mark.parametrize("scheme", ["testbed", "mixed", "area_64", "area_48_deep", "smoother", "testbed_retina",
                                    "retina", "retina_scaled", "area_256_shape"])
def test_cycles_match_oracle(ctx, scheme, plain):
    _run_parity(ctx, scheme, "default", plain, cycles=6)


# Specialised consumers each scheme's fused tufts reach once the flags are
# clean: 1 x 32 and 1 x 64 spiny stellate cells (1, 2), pyramidal cells of
# 8 x 32, 16 x 32 and 16 x 64 synapses (5, 6, 8); the mixed area's odd shapes
# mostly take the general consumer.
CLEAN_CONSUMERS = {"area_64": [1, 6], "area_48_deep": [1, 6], "area_256_shape": [2, 6], "testbed": [1],
                   "smoother": [1, 5], "mixed": [], "distal_1024": [1, 8]}
# Whether some tuft's footprint arrives as a tensor box: rows of a multiple of
# 16 bytes (64, 48 columns) do; the 24- and 40-column areas take the
# consumer-staged footprint.
CLEAN_TMA = {"area_64": True, "area_48_deep": True, "area_256_shape": True, "testbed": False, "smoother": False,
             "mixed": None, "distal_1024": True}


@pytest.mark.parametrize("scheme", sorted(CLEAN_CONSUMERS))
def test_clean_flag_cycles_match_oracle(ctx, scheme):
    """From scrambled states whose synapse flags carry only SYN_PREV_ACTIVE
    (the only bit bismit writes, cl/syns.cl:23-33), as in real runs: the fused
    path then serves its tufts with the compile-time specialised consumers."""
    _run_parity(ctx, scheme, "default", False, cycles=6, clean_flags=True, consumers=CLEAN_CONSUMERS[scheme],
                footprint_tma=CLEAN_TMA[scheme])


@pytest.mark.parametrize("plain", [True, False], ids=["plain", "fused"])
def test_bypassed_filters_match_oracle(ctx, plain):
    """With bypass_filters the frames go straight to the axons and no filter
    runs (AxonSpace::intake, src/cortex/axon_space.rs:516)."""
    _run_parity(ctx, "retina", "bypass_filters", plain, cycles=3)


def test_filtered_frames_from_device_match_oracle(ctx):
    """Per-cycle frames taken from device memory land in the filter chain's
    buffer as host-written ones do; a cycle with no new frame filters the
    stored one again."""
    import torch
    area = _area(ctx, "retina", settings_for())
    plan = area.plan
    slab = initial_slab(plan, 7, scramble_seed=11)
    area.write_slab(slab)
    area.set_cycle(0)
    fr = frames_for(plan, 4, 5, 0.05)
    dev = torch.from_numpy(np.ascontiguousarray(fr[:3])).to("cuda:0")
    torch.cuda.synchronize()
    area.cycle_frames_device(dev.data_ptr(), fr.shape[1], 3)
    area.cycle(1)
    ora = slab.copy()
    oracle.run(plan, ora, fr[:3], 3, start_cycle=0)
    oracle.run(plan, ora, None, 1, start_cycle=3)
    got = area.read_slab()
    assert np.array_equal(got, ora), diff_report(plan, got, ora)
    area.close()


@pytest.mark.parametrize("scheme", ["mixed", "retina"])
def test_host_frames_read_during_the_call_only(ctx, scheme):
    """bm_area_write_input reads the caller's bytes during the call only, even
    from pinned memory, whose copies are otherwise asynchronous: one pinned
    buffer, written twice before each cycle (the second frame wins) and
    spoiled right after each call, gives the oracle's state."""
    import ctypes as C
    import torch
    area = _area(ctx, scheme, settings_for())
    plan = area.plan
    slab = initial_slab(plan, 7, scramble_seed=11)
    area.write_slab(slab)
    area.set_cycle(0)
    n = 5
    fr = frames_for(plan, n + 1, 5, 0.05)
    flen = fr.shape[1]
    buf = torch.empty(flen, dtype=torch.uint8).pin_memory()
    lib = area.lib
    for k in range(n):
        for f in (fr[n - k], fr[k]):
            buf.copy_(torch.from_numpy(np.ascontiguousarray(f)))
            F.check(lib.bm_area_write_input(area.h, 0, C.c_void_p(buf.data_ptr()), C.c_size_t(flen)))
            buf.fill_(0xA5)
        area.cycle(1)
    ora = slab.copy()
    oracle.run(plan, ora, fr[:n], n, start_cycle=0)
    got = area.read_slab()
    assert np.array_equal(got, ora), diff_report(plan, got, ora)
    area.close()


@pytest.mark.parametrize("plain", [True, False], ids=["plain", "fused"])
@pytest.mark.parametrize("kind", ["bypass_inhib", "no_learning", "no_pyrs", "no_sscs"])
def test_settings_match_oracle(ctx, kind, plain):
    _run_parity(ctx, "mixed", kind, plain, cycles=3)


@pytest.mark.parametrize("plain", [True, False], ids=["plain", "fused"])
@pytest.mark.parametrize("scheme", ["testbed", "mixed", "area_64", "area_48_deep"])
def test_regrowth_matches_oracle(ctx, scheme, plain):
    """Cycles 198 to 201 with regrowth on: cycle 200 redraws every synapse whose
    strength is at or below the floor (Synapses::regrow,
    src/cortex/synapses.rs:411-501), the fused path's compiled gather offsets
    follow, and the cycles after it read the new sources."""
    plan, before, after = _run_parity(ctx, scheme, "regrowth", plain, cycles=4, start=198)
    moved = 0
    for name, off, n in buffers(plan):
        if name.endswith("syn_src_slc_ids") or name.endswith("syn_src_col_v_offs"):
            moved += int(np.count_nonzero(before[off:off + n] != after[off:off + n]))
    assert moved > 0


@pytest.mark.parametrize("plain", [True, False], ids=["plain", "fused"])
def test_unscrambled_long_run(ctx, plain):
    """From the grown state (no scrambling) for 40 cycles: learning moves the
    strengths and the pyramidal layer fires."""
    _run_parity(ctx, "area_64", "zero_strength", plain, cycles=40, scramble=False, active=0.02)


@pytest.mark.parametrize("plain", [True, False], ids=["plain", "fused"])
def test_caller_written_sources_match_oracle(ctx, plain):
    """Sources written by the caller (the reference's set_src_offs /
    set_src_slc test helpers, src/cortex/synapses.rs:589-600): any u8 slice id
    and any i8 offset, including ids past the last slice and offsets past the
    pool's reach, index exactly as axn_state_3d_safe does."""
    s = settings_for(plain=plain)
    area = _area(ctx, "area_48_deep", s)
    plan = area.plan
    slab = initial_slab(plan, 7, scramble_seed=3)
    rng = np.random.default_rng(17)
    for li in range(plan.n_layers):
        L = plan.layers[li]
        n = int(L.n_syns)
        idx = rng.choice(n, size=n // 50, replace=False)
        for name, lo, hi in (("syn_src_slc_ids", 0, 256), ("syn_src_col_v_offs", -128, 128),
                             ("syn_src_col_u_offs", -128, 128)):
            off = int(L.buf_off[F.BUF[name]])
            vals = rng.integers(lo, hi, idx.size).astype(np.int16).astype(np.uint8)
            slab[off + idx] = vals
    area.write_slab(slab)
    area.set_cycle(0)
    fr = frames_for(plan, 4, 5)
    ora = slab.copy()
    for k in range(4):
        area.write_input(fr[k])
        area.cycle(1)
        oracle.run(plan, ora, fr[k:k + 1], 1, start_cycle=k)
        dev = area.read_slab()
        assert np.array_equal(dev, ora), "cycle %d:\n%s" % (k, diff_report(plan, dev, ora))
    # Writing one source back into range through the buffer API is picked up too.
    L = plan.layers[1]
    area.write("syn_src_col_v_offs", np.zeros(64, np.int8), layer=1, offset=0)
    ora[int(L.buf_off[F.BUF["syn_src_col_v_offs"]]):][:64] = 0
    area.write_input(fr[0])
    area.cycle(1)
    oracle.run(plan, ora, fr[0:1], 1, start_cycle=4)
    dev = area.read_slab()
    assert np.array_equal(dev, ora), diff_report(plan, dev, ora)
    area.close()


def test_side_stream_follows_caller_sources(ctx):
    """The pyramidal distal tuft runs beside the spiny stellate chain while its
    sources stay in its pool; once the caller writes slice ids outside the
    pool it may read any slice, so it rejoins the chain; a slab restore with
    pool sources sends it back beside. (The plain form cycles a layer's tufts
    as one step, which reads the proximal tuft's spiny stellate axons and so
    always stays in the chain.)"""
    area = _area(ctx, "area_64", settings_for())
    grown = area.read_slab()
    n0 = area.side_steps()
    assert n0 >= 1
    li = next(i for i in range(area.plan.n_layers) if area.plan.layers[i].kind == F.BM_LYR_PYRAMIDAL)
    area.write("syn_src_slc_ids", np.array([250], np.uint8), layer=li,
               offset=int(area.plan.layers[li].n_syns) - 1)
    assert area.side_steps() < n0
    area.write_slab(grown)
    assert area.side_steps() == n0
    area.close()


@pytest.mark.parametrize("sampled", ["none", "pyramidal_axons", "ssc_axons"])
def test_front_stream_cycles_match_oracle(ctx, sampled):
    """The spiny stellate tuft and inhibition run on the front stream, each
    cycle's beside the previous cycle's pyramidal steps, with host frames
    (one call per cycle) and with a block of device frames (one call for
    several cycles). A sampler of the pyramidal axons leaves the front stream
    in use and gets every cycle's frame; one of the spiny stellate axons, which
    the front steps write, turns it off. Whole slabs equal the oracle's."""
    import torch
    area = _area(ctx, "area_256_shape", settings_for())
    plan = area.plan
    slab = initial_slab(plan, 7, scramble_seed=23, clean_flags=True)
    area.write_slab(slab)
    area.set_cycle(0)
    ssc = next(i for i in range(plan.n_layers) if plan.layers[i].kind == F.BM_LYR_SPINY_STELLATE)
    pyr = next(i for i in range(plan.n_layers) if plan.layers[i].kind == F.BM_LYR_PYRAMIDAL)
    smp = None if sampled == "none" else area.sampler("axons", pyr if sampled == "pyramidal_axons" else ssc)
    assert area.front_steps() == (0 if sampled == "ssc_axons" else 2)
    fr = frames_for(plan, 8, 5, 0.05)
    ora = slab.copy()
    for c in range(3):
        area.write_input(fr[c])
        area.cycle(1)
        oracle.run(plan, ora, fr[c:c + 1], 1, start_cycle=c)
        if smp is not None:
            cyc, frame = smp.recv(wait_for_frame=True)
            assert cyc == c
    dev = torch.from_numpy(np.ascontiguousarray(fr[3:])).to("cuda:0")
    torch.cuda.synchronize()
    area.cycle_frames_device(dev.data_ptr(), fr.shape[1], 5)
    oracle.run(plan, ora, fr[3:], 5, start_cycle=3)
    got = area.read_slab()
    assert np.array_equal(got, ora), diff_report(plan, got, ora)
    assert area.cycle_count() == 8
    if smp is not None:
        smp.close()
    area.close()


def test_device_error_bits_clear(ctx):
    import ctypes
    area = _area(ctx, "area_64", settings_for())
    area.cycle(3)
    bits = ctypes.c_uint32(99)
    assert area.lib.bm_area_device_errors(area.h, ctypes.byref(bits)) == 0
    assert bits.value == 0
    area.close()


def test_cortex_builder_end_to_end():
    """The builder surface: Cortex.builder(..).ca_settings(..).build(), input,
    cycle, output, against the oracle on the same grown state."""
    from bismit_b200 import Cortex, configs
    lmaps, areas, act = configs.workload("area_64")
    cx = Cortex.builder(lmaps, areas).ca_settings(configs.bench_settings()).seed(3).build()
    a = cx.area("v1")
    slab = a.read_slab()
    fr = configs.frames(5, a.input_len(), act, 9)
    for k in range(5):
        a.write_input(fr[k])
        cx.cycle()
    out = a.read_output()
    oracle.run(a.plan, slab, fr, 5, 0)
    o = a.plan.outputs[0]
    assert np.array_equal(out, slab[a.plan.axon_off + o.axn_idz: a.plan.axon_off + o.axn_idz + o.len])
    assert np.array_equal(a.read_slab(), slab)
    assert a.cycle_count() == 5
    cx.close()


def test_buffer_io_bounds(ctx):
    area = _area(ctx, "area_64", settings_for())
    with pytest.raises(F.BismitError):
        area.read("syn_states", layer=0, offset=int(area.plan.layers[0].n_syns), length=1)
    with pytest.raises(F.BismitError):
        area.write_input(np.zeros(area.input_len() + 1, np.uint8))
    x = np.arange(64, dtype=np.int8)
    area.write("syn_strengths", x, layer=1, offset=100)
    assert np.array_equal(area.read("syn_strengths", layer=1, offset=100, length=64), x)
    area.close()
