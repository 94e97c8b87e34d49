"""Serving (bm_server_*): sessions arriving over time, admitted by a memory
budget that forces some to wait, cycled together as they have frames. Every
session's state after its last frame must be byte-identical to the same
session run alone (tolerance: exact), and its outputs must be the alone
run's outputs.
"""
import time

import numpy as np
import pytest

from bismit_b200 import configs, cortex, map as M, plan_of

# (side, depth, dens, syns, frames, arrival tick)
SESSIONS = [(32, 1, 8, 16, 5, 0), (48, 2, 16, 32, 7, 0), (40, 1, 8, 64, 4, 0),
            (64, 3, 16, 16, 6, 1), (32, 2, 8, 32, 3, 2), (56, 1, 16, 64, 5, 3)]


def _desc(side, depth, dens, syns):
    lmaps, areas = configs.instance_area(side, depth, dens, syns)
    return M.area_desc("v1", lmaps, areas, configs.bench_settings())


def _footprint(plan):
    b = int(plan.slab_bytes) + 2 * int(plan.n_syns_total) + 4096 + 272
    return (b + 0xFFFFF) & ~0xFFFFF


@pytest.mark.gpu
def test_sessions_in_the_mix_match_sessions_alone():
    ctx = cortex._Ctx(0)
    descs = [_desc(*s[:4]) for s in SESSIONS]
    plans = [plan_of(d, 100 + k) for k, d in enumerate(descs)]
    frames = [configs.frames(s[4], int(p.inputs[0].len), 0.03, 200 + k) for k, (s, p) in enumerate(zip(SESSIONS, plans))]
    budget = sum(sorted(_footprint(p) for p in plans)[-3:])   # about three sessions at a time
    srv = cortex.Server(ctx, budget)
    sid = {}
    final, outs = {}, {k: [] for k in range(len(SESSIONS))}
    tick = 0
    deadline = time.monotonic() + 120
    while len(final) < len(SESSIONS):
        for k, s in enumerate(SESSIONS):
            if s[5] == tick:
                sid[k] = srv.open(descs[k], 100 + k)
                srv.submit(sid[k], frames[k])
        n = srv.tick()
        for k in list(sid):
            if k in final:
                continue
            out, done = srv.read_output(sid[k], int(plans[k].outputs[0].len))
            if done > len(outs[k]):
                outs[k].append(out)
            if done == SESSIONS[k][4]:
                final[k] = srv.session_slab(sid[k], plans[k].slab_bytes)
                srv.close_session(sid[k])
        st = srv.stats()
        assert st["used_bytes"] <= budget
        tick += 1
        assert time.monotonic() < deadline, "sessions never drained"
        if n == 0:
            time.sleep(0.001)   # areas are being built off the tick path
    st = srv.stats()
    assert st["frames"] == sum(s[4] for s in SESSIONS)
    assert st["p99_ms"] >= st["p50_ms"] > 0
    # The slowest tick is described: its device time, number and sessions.
    assert st["tick_max_ms"] >= st["tick_p99_ms"] > 0
    assert st["tick_max_no"] < st["ticks"] and 1 <= st["tick_max_members"] <= len(SESSIONS)
    assert st["tick_max_queue_ms"] >= 0
    srv.close()
    # Each session alone.
    for k, d in enumerate(descs):
        a = cortex.CorticalArea(ctx, d, 100 + k)
        for c in range(SESSIONS[k][4]):
            a.write_input(frames[k][c])
            a.cycle(1)
            assert np.array_equal(a.read_output(), outs[k][c]), "session %d, frame %d output" % (k, c)
        assert np.array_equal(a.read_slab(), final[k]), "session %d state differs from its run alone" % k
        a.close()
    ctx.close()


@pytest.mark.gpu
def test_admission_waits_for_memory():
    ctx = cortex._Ctx(0)
    d = _desc(48, 2, 16, 32)
    p = plan_of(d, 1)
    srv = cortex.Server(ctx, _footprint(p) + 1024)   # room for one session
    a = srv.open(d, 1)
    b = srv.open(d, 2)
    fr = configs.frames(2, int(p.inputs[0].len), 0.03, 9)
    srv.submit(a, fr)
    srv.submit(b, fr)
    srv.close_session(a)
    srv.close_session(b)
    deadline = time.monotonic() + 60
    while srv.stats()["frames"] < 4:
        if srv.tick() == 0:
            time.sleep(0.001)   # areas are being built off the tick path
        st = srv.stats()
        assert st["resident"] <= 1 and st["used_bytes"] <= _footprint(p) + 1024
        assert time.monotonic() < deadline
    srv.close()
    ctx.close()


@pytest.mark.gpu
def test_a_failing_session_is_dropped_and_the_others_match_alone():
    """A session whose area ends a cycle with device error bits (here a
    bounded wait made to run out through the fault hook, with a 1 ms limit)
    is dropped: one tick reports BM_ERR_TIMEOUT, reading its output reports
    it too, and the other sessions finish with the bytes they have alone. A
    cancelled session leaves with its queued frames discarded."""
    import ctypes
    from bismit_b200 import _ffi as F
    ctx = cortex._Ctx(0)
    shapes = [(48, 2, 16, 32), (64, 1, 8, 64), (40, 2, 8, 16), (32, 1, 16, 16)]
    n_frames = 8
    descs = [_desc(*s) for s in shapes]
    plans = [plan_of(d, 300 + k) for k, d in enumerate(descs)]
    frames = [configs.frames(n_frames, int(p.inputs[0].len), 0.03, 400 + k) for k, p in enumerate(plans)]
    srv = cortex.Server(ctx, 0)
    sid = [srv.open(d, 300 + k) for k, d in enumerate(descs)]
    for k in range(len(sid)):
        srv.submit(sid[k], frames[k])
    FAIL, CANCEL = 1, 3
    deadline = time.monotonic() + 120
    while srv.stats()["frames"] < len(sid):   # every session resident and cycling
        if srv.tick() == 0:
            time.sleep(0.001)
        assert time.monotonic() < deadline
    h = ctypes.c_void_p()
    F.check(srv.lib.bm_server_session_area(srv.h, sid[FAIL], ctypes.byref(h)))
    F.check(srv.lib.bm_area_set_wait_limit(h, 1000))
    F.check(srv.lib.bm_area_inject_stall(h, 1))
    srv.cancel_session(sid[CANCEL])
    reported = 0
    final = {}
    while len(final) < len(sid) - 2:
        try:
            srv.tick()
        except F.BismitError as e:
            assert e.code == F.BM_ERR_TIMEOUT and "dropped" in str(e)
            reported += 1
        for k in (0, 2):
            if k in final:
                continue
            _out, done = srv.read_output(sid[k], int(plans[k].outputs[0].len))
            if done == n_frames:
                final[k] = srv.session_slab(sid[k], plans[k].slab_bytes)
                srv.close_session(sid[k])
        assert time.monotonic() < deadline
    assert reported == 1
    with pytest.raises(F.BismitError) as e:
        srv.read_output(sid[FAIL], int(plans[FAIL].outputs[0].len))
    assert e.value.code == F.BM_ERR_TIMEOUT
    assert srv.stats()["failed"] == 1
    srv.close()
    for k in final:
        a = cortex.CorticalArea(ctx, descs[k], 300 + k)
        for c in range(n_frames):
            a.write_input(frames[k][c])
            a.cycle(1)
        assert np.array_equal(a.read_slab(), final[k]), "session %d differs from its run alone" % k
        a.close()
    ctx.close()
