"""The bench's whole-cycle byte count: the learning criterion it counts on the
device (bench.pyr_learners, and spiny stellate cells with a non-zero axon)
must cover every synapse whose strength learning changes. Checked over oracle
cycles on the CPU (ssc_mtp_simple, cl/bismit.cl:888-915; tft_dst_mtp,
cl/bismit.cl:1195-1268)."""
import numpy as np

import bench
import oracle
from bismit_b200 import _ffi as F, configs, map as M, plan_of


def test_learning_criterion_covers_every_changed_strength():
    lmaps, areas, _ = configs.workload("area_64")
    desc = M.area_desc("v1", lmaps, areas, configs.bench_settings())
    plan = plan_of(desc, 3)
    slab = np.zeros(int(plan.slab_bytes), np.uint8)
    oracle.grow(plan, slab, 3, desc.init_flags)
    fr = configs.frames(8, int(plan.inputs[0].len), 0.05, 1)
    B = F.BUF
    learned = {F.BM_LYR_SPINY_STELLATE: 0, F.BM_LYR_PYRAMIDAL: 0}
    for k in range(len(fr)):
        before = slab.copy()
        oracle.run(plan, slab, fr[k:k + 1], 1, start_cycle=k)
        for i in range(plan.n_layers):
            L = plan.layers[i]
            a0 = int(plan.axon_off) + int(L.axn_idz)
            ax = slab[a0:a0 + L.cells]
            so, sl = int(L.buf_off[B["syn_strengths"]]), int(L.buf_len[B["syn_strengths"]])
            changed = np.nonzero(slab[so:so + sl] != before[so:so + sl])[0]
            covered = np.zeros(sl, bool)
            if L.kind == F.BM_LYR_SPINY_STELLATE:
                spt = int(L.tufts[0].syns_per_tft)
                for c in np.nonzero(ax)[0]:
                    covered[c * spt:(c + 1) * spt] = True
            elif L.kind == F.BM_LYR_PYRAMIDAL:
                T = [L.tufts[t] for t in range(L.n_tufts) if L.tufts[t].den_kind == F.BM_DEN_DISTAL][0]
                fo = int(L.buf_off[B["cel_flag_sets"]])
                ro = int(L.buf_off[B["tft_prev_best_den_states_raw"]]) + int(T.cel_idz)
                io = int(L.buf_off[B["tft_prev_best_den_ids"]]) + int(T.cel_idz)
                spd, spt = int(T.syns_per_den), int(T.syns_per_tft)
                ids = slab[io:io + L.cells]
                for c in np.nonzero(bench.pyr_learners(before[fo:fo + L.cells], ax, slab[ro:ro + L.cells]))[0]:
                    z = int(ids[c]) * spd + int(c) * spt + int(T.syn_idz)
                    covered[z:z + spd] = True
            else:
                continue
            assert covered[changed].all(), "cycle %d layer %d: a changed strength outside the counted runs" % (k, i)
            learned[L.kind] += len(changed)
    # Both learning rules ran.
    assert learned[F.BM_LYR_SPINY_STELLATE] > 0 and learned[F.BM_LYR_PYRAMIDAL] > 0


def test_cycle_bytes_of_area_256():
    """7 B a synapse, 4 a dendrite, 12 a pyramidal cell-tuft, 4 a cell, the
    frame and 3 a learning synapse: about 1.95 GB for 256x256 columns."""
    lmaps, areas, _ = configs.workload("area_256")
    plan = plan_of(M.area_desc("v1", lmaps, areas, configs.bench_settings()), 0)
    b0 = bench.cycle_bytes(plan, int(plan.inputs[0].len), 0)
    assert bench.cycle_bytes(plan, int(plan.inputs[0].len), 1000) - b0 == 3000
    assert 1.90e9 < b0 < 1.96e9
