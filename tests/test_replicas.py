"""Multi-rank replicas on the host (gloo, world size 2): each rank runs an
independent replica of an area (its own seeds), with no collective on the
data path; the job's time is the slowest rank's and its work the sum of all
ranks'. Each rank's bytes must equal a single-process run with that rank's
seeds. Runs the oracle as the per-rank workload (no GPU)."""
import hashlib
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import oracle
from bismit_b200 import configs, map as M, plan_of, replicas

WS = 2
CYCLES = 2


def _desc():
    lmaps, areas = configs.testbed_area(16)
    return M.area_desc("v1", lmaps, areas, configs.bench_settings())


def _replica(rank):
    """The slab digest and synapse count of rank `rank`'s replica after CYCLES cycles."""
    seed = replicas.replica_seed(7, rank)
    plan = plan_of(_desc(), seed)
    slab = np.zeros(int(plan.slab_bytes), np.uint8)
    oracle.grow(plan, slab, seed, 0)
    fr = configs.frames(CYCLES, int(plan.inputs[0].len), 0.05, replicas.frame_seed(7, rank))
    oracle.run(plan, slab, fr, CYCLES, 0)
    return hashlib.sha256(slab.tobytes()).hexdigest(), int(plan.n_syns_total)


def _worker(rank, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WS, timeout=datetime.timedelta(seconds=60))
    digest, n_syn = _replica(rank)
    ms = 10.0 + rank   # each rank's "time"
    q.put((rank, digest, n_syn, replicas.max_over_ranks(ms), replicas.sum_over_ranks(n_syn),
           replicas.job_throughput(n_syn, ms)))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_replicas_are_independent_and_timed_by_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in range(WS)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(WS):
        r = q.get(timeout=120)
        got[r[0]] = r
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    digests = {r: got[r][1] for r in got}
    assert digests[0] != digests[1]                      # distinct replicas
    for r in range(WS):
        d, n = _replica(r)                               # single-process run of that rank's replica
        assert got[r][1] == d
        assert got[r][3] == 11.0                         # max over ranks
        assert got[r][4] == WS * n                       # sum over ranks
        assert abs(got[r][5] - WS * n / 0.011) < 1e-6 * WS * n / 0.011
    assert replicas.replica_seed(7, 0) == 7              # rank 0 = a single-process run
