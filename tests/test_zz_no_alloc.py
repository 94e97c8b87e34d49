"""bm_tuft_cycle_static, the entry point that allocates no device memory,
against bm_area_cycle on the same state.

With the spatial layers switched off (CorticalAreaSettings::disable_sscs),
the first layer of a cycle is the pyramidal layer, so its tuft stages
read exactly the state the caller wrote before the cycle. Nothing later in
the cycle writes the buffers those stages produce: the pyramidal cycle writes
cell states, learning writes strengths and cell flags, the outputs write axons.
Each tuft's synapse, dendrite and cell-tuft outputs after bm_area_cycle are
therefore the outputs the static entry point must produce on a copy of the
pre-cycle state. The test runs two steps in a row, each calling every tuft of
the layer in a different order, so each call finds the shared scratch holding
the previous call's contents.

This file is named to be collected last; it passes alone in a fresh process
too (the first call on the device does the one-time set-up).
"""
import ctypes as C

import numpy as np
import pytest

from bismit_b200 import _ffi as F, cortex
from helpers import desc_of, frames_for, scramble, settings_for

SYN_OUT = ("syn_states", "syn_flag_sets")
DEN_OUT = ("den_states_raw", "den_states", "den_activities")
TFT_OUT = ("tft_best_den_ids", "tft_best_den_states_raw", "tft_best_den_states", "tft_states",
           "tft_prev_best_den_ids", "tft_prev_best_den_states_raw", "tft_prev_best_den_states",
           "tft_prev_states")
MAX_SYNS = 1 << 22


def _out_ranges(plan, li, t):
    """(name, slab offset, length) of every buffer range the tuft stage writes."""
    L = plan.layers[li]
    T = L.tufts[t]
    cells = int(L.cells)
    out = []
    for n in SYN_OUT:
        out.append((n, int(L.buf_off[F.BUF[n]]) + int(T.syn_idz), cells * int(T.syns_per_tft)))
    for n in DEN_OUT:
        out.append((n, int(L.buf_off[F.BUF[n]]) + int(T.den_idz), cells * int(T.dens_per_tft)))
    if L.kind == F.BM_LYR_PYRAMIDAL:
        for n in TFT_OUT:
            out.append((n, int(L.buf_off[F.BUF[n]]) + int(T.cel_idz), cells))
    return out


def _static(lib, plan, li, t, slab_ptr, cycle, err_ptr, stream):
    return lib.bm_tuft_cycle_static(C.byref(plan), li, t, C.c_void_p(slab_ptr), C.c_uint64(cycle),
                                    C.c_void_p(err_ptr), C.c_void_p(stream))


@pytest.mark.gpu
@pytest.mark.parametrize("flags", ["clean", "foreign"])
def test_static_tuft_cycle_matches_area_cycle(flags):
    """With clean flags (only SYN_PREV_ACTIVE, as in real runs) the calls run
    the tiled kernel with its specialised consumers and the gather offsets in
    the shared scratch; with foreign flag bits, the form that streams flags
    through. Device free memory is unchanged across the calls after the
    first."""
    import torch

    ctx = cortex._Ctx(0)
    desc = desc_of("area_48_deep", settings_for("no_sscs"))
    a = cortex.CorticalArea(ctx, desc, 7)    # runs bm_area_cycle
    b = cortex.CorticalArea(ctx, desc, 7)    # its slab stands in for the caller's own memory
    plan = a.plan
    lib = a.lib
    li = next(int(plan.cycle_order[k]) for k in range(plan.n_cycle_order)
              if not plan.layers[int(plan.cycle_order[k])].tags & F.BM_TAG_SPATIAL)
    L = plan.layers[li]
    assert L.kind == F.BM_LYR_PYRAMIDAL and L.n_tufts >= 2
    tufts = list(range(int(L.n_tufts)))
    for t in tufts:
        assert int(L.cells) * int(L.tufts[t].syns_per_tft) <= MAX_SYNS
    ptr = C.c_void_p()
    F.check(lib.bm_area_slab_ptr(b.h, C.byref(ptr)))
    err = torch.full((len(tufts),), 0xFF, dtype=torch.int32, device="cuda:0")
    stream = torch.cuda.Stream(device=0)

    slab = a.read_slab()
    scramble(plan, slab, 11, clean_flags=flags == "clean")
    a.write_slab(slab)
    a.set_cycle(0)
    forms = [a.tuft_form(li, t) for t in tufts]
    assert any(f["tiled"] for f in forms), forms
    if flags == "clean":
        assert all(not f["flags_foreign"] for f in forms) and any(f["consumer"] for f in forms), forms
    else:
        assert all(f["flags_foreign"] for f in forms if f["fused"]), forms
    fr = frames_for(plan, 2, 5, 0.05)
    for k, order in enumerate((tufts[::-1], tufts)):
        b.write_slab(a.read_slab())
        if fr is not None:
            a.write_input(fr[k])
            b.write_input(fr[k])
        before = b.read_slab()
        a.cycle(1)
        want = a.read_slab()
        torch.cuda.synchronize()
        stream.wait_stream(torch.cuda.current_stream())   # err's fill comes first
        free0 = torch.cuda.mem_get_info(0)[0]
        for j, t in enumerate(order):
            rc = _static(lib, plan, li, t, ptr.value, k, err.data_ptr() + 4 * j, stream.cuda_stream)
            assert rc == F.BM_OK, lib.bm_last_error().decode()
        stream.synchronize()
        if k > 0:   # the first call on the device may load the library's module
            assert torch.cuda.mem_get_info(0)[0] == free0
        got = b.read_slab()
        assert err.tolist() == [0] * len(tufts)
        written = np.zeros(got.size, bool)
        for t in tufts:
            for name, off, n in _out_ranges(plan, li, t):
                assert np.array_equal(got[off:off + n], want[off:off + n]), \
                    "step %d tuft %d %s: %d bytes differ" % (k, t, name, int((got[off:off + n] != want[off:off + n]).sum()))
                written[off:off + n] = True
        # Nothing outside the tufts' output ranges changed.
        assert np.array_equal(got[~written], before[~written]), "step %d: write outside the tuft outputs" % k
        err.fill_(0xFF)
    assert a.cycle_count() == 2
    a.close()
    b.close()
    ctx.close()


@pytest.mark.gpu
def test_static_rejects_tufts_outside_the_fused_shapes():
    ctx = cortex._Ctx(0)
    a = cortex.CorticalArea(ctx, desc_of("area_64", settings_for()), 7)
    ptr = C.c_void_p()
    F.check(a.lib.bm_area_slab_ptr(a.h, C.byref(ptr)))
    # Layer 1, tuft 0 is the one-synapse proximal tuft.
    assert _static(a.lib, a.plan, 1, 0, ptr.value, 0, 0, 0) == F.BM_ERR_UNSUPPORTED
    a.close()
    ctx.close()


def test_static_rejects_bad_arguments_before_touching_the_device():
    """Size and range checks come first: no device is needed to see them."""
    from bismit_b200 import configs, map as M, plan_of
    lmaps, areas, _ = configs.workload("area_256")
    plan = plan_of(M.area_desc("v1", lmaps, areas, configs.bench_settings()), 7)
    lib = F.lib()
    fake = 1 << 40   # never dereferenced: every call below is rejected first
    li = next(i for i in range(plan.n_layers) if plan.layers[i].kind == F.BM_LYR_PYRAMIDAL)
    L = plan.layers[li]
    big = max(range(L.n_tufts), key=lambda t: L.tufts[t].syns_per_tft)
    assert int(L.cells) * int(L.tufts[big].syns_per_tft) > MAX_SYNS
    assert _static(lib, plan, li, big, fake, 0, 0, 0) == F.BM_ERR_INVALID
    assert "at most 4194304" in lib.bm_last_error().decode()
    assert _static(lib, plan, plan.n_layers, 0, fake, 0, 0, 0) == F.BM_ERR_INVALID
    assert _static(lib, plan, li, L.n_tufts, fake, 0, 0, 0) == F.BM_ERR_INVALID
    assert _static(lib, plan, li, 0, 0, 0, 0, 0) == F.BM_ERR_INVALID
