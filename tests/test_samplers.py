"""Samplers (bm_sampler_*): per-cycle readback through a one-frame channel,
CorticalArea::sampler (src/cortex/cortical_area.rs:809-880,1017-1284) with
the tract channel's rules (src/subcortex/tract_channel.rs:400-488):
  * a frame is sent after a cycle when the receiver has taken the last one;
  * otherwise the new frame is skipped, or with backpressure the cycling call
    waits for the receiver;
  * recv takes the unread frame, or waits for one, or returns none.
Frames are compared byte for byte with the area's own buffers read after the
same cycle.
"""
import threading
import time

import numpy as np
import pytest

from bismit_b200 import _ffi as F, configs, cortex, map as M
from helpers import desc_of, frames_for, scramble, settings_for

pytestmark = pytest.mark.gpu

# (sampler kind, area read buffer name)
KINDS = [("soma_states", "cel_states"), ("syn_strengths", "syn_strengths"), ("den_states", "den_states"),
         ("tuft_best_den_ids", "tft_best_den_ids"), ("syn_flag_sets", "syn_flag_sets")]


@pytest.fixture(scope="module")
def ctx():
    c = cortex._Ctx(0)
    yield c
    c.close()


def _area(ctx, seed=7):
    a = cortex.CorticalArea(ctx, desc_of("mixed", settings_for()), seed)
    slab = a.read_slab()
    scramble(a.plan, slab, 3)
    a.write_slab(slab)
    a.set_cycle(0)
    return a


def _pyr_layer(a):
    for i in range(a.plan.n_layers):
        if a.plan.layers[i].kind == F.BM_LYR_PYRAMIDAL:
            return i
    raise AssertionError("no pyramidal layer")


def test_frames_equal_the_buffers_after_each_cycle(ctx):
    a = _area(ctx)
    li = _pyr_layer(a)
    smp = {k: a.sampler(k, li) for k, _ in KINDS}
    ax = a.sampler("axons")                     # every axon of the area
    ax_l = a.sampler("axons", li)                # the layer's slices
    fr = frames_for(a.plan, 4, 5, 0.05)
    L = a.plan.layers[li]
    k0 = int(L.base_axn_slc)
    a0 = int(a.plan.slc_axn_idz[k0])
    n_l = sum(int(a.plan.slc_v_size[k]) * int(a.plan.slc_u_size[k]) for k in range(k0, k0 + int(L.depth)))
    for c in range(4):
        a.write_input(fr[c])
        a.cycle(1)
        for kind, buf in KINDS:
            got = smp[kind].recv()
            assert got is not None, kind
            cyc, frame = got
            assert cyc == c
            assert np.array_equal(frame, a.read(buf, li)), kind
            assert smp[kind].recv() is None   # taken
        cyc, frame = ax.recv()
        axons = a.read("axon_states")
        assert cyc == c and np.array_equal(frame, axons)
        cyc, frame = ax_l.recv()
        assert cyc == c and np.array_equal(frame, axons[a0:a0 + n_l])
    a.close()


def test_unread_frame_is_kept_and_new_ones_skipped(ctx):
    a = _area(ctx)
    li = _pyr_layer(a)
    s = a.sampler("soma_states", li)
    fr = frames_for(a.plan, 3, 5, 0.05)
    a.write_input(fr[0])
    a.cycle(1)
    first = a.read("cel_states", li)
    for c in (1, 2):
        a.write_input(fr[c])
        a.cycle(1)
    cyc, frame = s.recv()
    assert cyc == 0 and np.array_equal(frame, first)
    assert s.recv() is None
    assert s.stats() == {"sent": 1, "skipped": 2}
    a.close()


def test_backpressure_delivers_every_cycle_in_order(ctx):
    """With backpressure every cycle's frame reaches a receiver thread that
    takes them slowly; a twin area cycled alone gives the expected bytes."""
    a, twin = _area(ctx), _area(ctx)
    li = _pyr_layer(a)
    s = a.sampler("den_states", li, backpressure=True)
    s.set_timeout(20000)   # a stuck receiver fails the test instead of hanging it
    n = 6
    fr = frames_for(a.plan, n, 5, 0.05)
    got = []

    def receive():
        for _ in range(n):
            time.sleep(0.02)
            got.append(s.recv(wait_for_frame=True))

    th = threading.Thread(target=receive)
    th.start()
    expect = []
    for c in range(n):
        a.write_input(fr[c])
        a.cycle(1)
        twin.write_input(fr[c])
        twin.cycle(1)
        expect.append(twin.read("den_states", li))
    th.join(timeout=60)
    assert not th.is_alive()
    assert [g[0] for g in got] == list(range(n))
    for (cyc, frame), e in zip(got, expect):
        assert np.array_equal(frame, e), cyc
    assert s.stats() == {"sent": n, "skipped": 0}
    a.close()
    twin.close()


def test_backpressure_wait_is_bounded(ctx):
    a = _area(ctx)
    s = a.sampler("soma_states", _pyr_layer(a), backpressure=True)
    s.set_timeout(100)
    a.cycle(1)                 # sent
    with pytest.raises(F.BismitError) as e:
        a.cycle(1)             # the first frame is unread: waits 100 ms, then gives up
    assert e.value.code == F.BM_ERR_TIMEOUT
    assert s.recv() is not None
    assert s.set_backpressure(False) is True
    a.cycle(2)                 # no backpressure: sent, then skipped
    assert s.stats()["skipped"] >= 1
    a.close()


def test_recv_wait_is_bounded(ctx):
    a = _area(ctx)
    s = a.sampler("soma_states", _pyr_layer(a))
    s.set_timeout(50)
    with pytest.raises(F.BismitError) as e:
        s.recv(wait_for_frame=True)
    assert e.value.code == F.BM_ERR_TIMEOUT
    a.close()


def test_samplers_follow_batched_cycles(ctx):
    descs = [M.area_desc("v1", *configs.instance_area(side, 1, 8, 16), configs.bench_settings())
             for side in (32, 48)]
    areas = []
    for k, d in enumerate(descs):
        a = cortex.CorticalArea(ctx, d, 5 + k)
        slab = a.read_slab()
        scramble(a.plan, slab, 40 + k)
        a.write_slab(slab)
        a.set_cycle(0)
        areas.append(a)
    li = _pyr_layer(areas[1])
    s = areas[1].sampler("syn_states", li)
    batch = cortex.Batch(ctx, areas)
    for c in range(3):
        batch.cycle(1)
        cyc, frame = s.recv()
        assert cyc == c
        assert np.array_equal(frame, areas[1].read("syn_states", li))
    batch.close()
    for a in areas:
        a.close()


class ChannelModel:
    """The tract channel of src/subcortex/tract_channel.rs:400-488 restated
    for one sender and one receiver polling from the same thread (recv with
    wait_for_frame false): `send` sets the ready flag; if it was already set
    the frame is skipped (without backpressure) or the sender waits (with it,
    which a single-threaded script never reaches); `recv` takes the waiting
    frame and clears the flag, or returns none. The library's channel also
    serves a receiver that waits for a frame, which the reference leaves
    untested (its direct hand-off keeps the ready flag set, :420-427)."""

    def __init__(self, backpressure):
        self.backpressure = backpressure
        self.ready = False
        self.frame = None
        self.sent = self.skipped = 0

    def send(self, cycle):
        if self.ready:
            assert not self.backpressure, "a single-threaded script would block here"
            self.skipped += 1
            return
        self.ready = True
        self.frame = cycle
        self.sent += 1

    def recv(self):
        if not self.ready:
            return None
        self.ready = False
        return self.frame


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_channel_matches_a_restatement_of_the_reference_channel(ctx, seed):
    """A seeded script of cycles, polls and backpressure switches drives the
    area's sampler and the restated channel side by side: the same frames
    (by cycle and content) come out, with the same sent and skipped counts.
    Backpressure is only on while the receiver has taken the last frame, so
    no send of the script blocks."""
    rng = np.random.default_rng(seed)
    a = _area(ctx)
    li = _pyr_layer(a)
    smp = a.sampler("soma_states", li)
    model = ChannelModel(False)
    fr = frames_for(a.plan, 40, 9, 0.05)
    states = {}
    c = 0
    for _ in range(120):
        op = rng.integers(0, 3)
        if op == 0 and c < len(fr):
            if not model.ready and rng.random() < 0.3:
                want = not model.backpressure
                assert smp.set_backpressure(want) == model.backpressure
                model.backpressure = want
            elif model.ready and model.backpressure:
                assert smp.set_backpressure(False) is True
                model.backpressure = False
            a.write_input(fr[c])
            a.cycle(1)
            states[c] = a.read("cel_states", layer=li)
            model.send(c)
            c += 1
        else:
            got = smp.recv(False)
            want = model.recv()
            if want is None:
                assert got is None
            else:
                assert got is not None and got[0] == want
                assert np.array_equal(got[1], states[want])
    st = smp.stats()
    assert (st["sent"], st["skipped"]) == (model.sent, model.skipped)
    assert model.skipped > 0 and model.sent > 0
    smp.close()
    a.close()
