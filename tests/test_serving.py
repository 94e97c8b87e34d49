"""Serving (bm_server_*): sessions arriving over time, admitted by a memory
budget that forces some to wait, cycled together as they have frames. Every
session's state after its last frame must be byte-identical to the same
session run alone (tolerance: exact), and its outputs must be the alone
run's outputs.
"""
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
        assert tick < 200, "sessions never drained"
    st = srv.stats()
    assert st["frames"] == sum(s[4] for s in SESSIONS)
    assert st["p99_ms"] >= st["p50_ms"] > 0
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
    ticks = 0
    while srv.stats()["frames"] < 4:
        srv.tick()
        st = srv.stats()
        assert st["resident"] <= 1
        ticks += 1
        assert ticks < 20
    srv.close()
    ctx.close()
