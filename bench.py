"""Benchmark: synapse-cycles/s of bismit's cortical cycle with learning on B200.

One step = one full cycle (intake, spiny stellate layer with inhibition and
learning, pyramidal layer with column inhibition and learning) of one area over
one input frame. Default workload: area_256 (256 x 256 columns, 272,629,760
synapses), the reference's single-area bandwidth configuration.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload area_256] [--path fused|plain]

With N > 1 (launched by torch.distributed.run) every rank runs an independent
replica of the area (no collective on the data path: the areas are
independent), timing is the max over ranks and `value` counts all ranks'
synapses ("scaling": "weak").
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "synapse-cycles/s incl. learning (bit-exact)"
UNIT = "synapse-cycles/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="area_256")
    ap.add_argument("--path", default="fused", choices=["fused", "plain"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--parity-cycles", type=int, default=3,
                    help="cycles of the headline area compared with bismit's kernels on the host (0: skip)")
    ap.add_argument("--cpu-sample-seconds", type=float, default=12.0)
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-instances measurement")
    ap.add_argument("--batch-instances", type=int, default=64)
    ap.add_argument("--no-serving", action="store_true", help="skip the serving measurement")
    ap.add_argument("--no-hierarchy", action="store_true", help="skip the three-area hierarchy measurement")
    ap.add_argument("--no-small", action="store_true", help="skip the 64 x 64 area measurement")
    ap.add_argument("--serve-sessions", type=int, default=64)
    ap.add_argument("--serve-rate", type=float, default=200.0, help="mean session arrivals per second (Poisson)")
    ap.add_argument("--serve-budget-gb", type=float, default=8.0)
    ap.add_argument("--profile-run", default=None, choices=["area", "batched", "hierarchy", "encoders"],
                    help="only W warm-up and K timed cycles of the workload (area: --workload through the plain "
                         "cycling call, --workload also smoother or retina; batched: the --batch-instances batch, "
                         "autotuned, graph replay; hierarchy: the three-area cortex with its tracts, autotuned, "
                         "graph replay; encoders: rounds of every device encoder into 64 frames of 256 x 256), "
                         "no soak, arms or baselines: a short launch sequence for a profiler's launch list")
    ap.add_argument("--regrowth", action="store_true", help="--profile-run area: with synapse regrowth on")
    ap.add_argument("--autotune-cache", default=None,
                    help="--profile-run batched or hierarchy: the autotuner's cache file (choices found there are applied "
                         "without trial launches; new ones are added)")
    return ap.parse_args()


def dist_env():
    from bismit_b200.replicas import dist_env as env
    return env()


def workload_config(name, n_syn):
    """The workload of one area, as both arms print it (the same keys and
    values; with N GPUs each rank runs one such area)."""
    from bismit_b200 import configs
    side, s, d, pd, ps, pr, act = configs.WORKLOADS[name]
    return {
        "workload": name,
        "columns": "%dx%d" % (side, side),
        "spiny_stellate": "1 tuft x 1 dendrite x %d synapses, reach 6" % s,
        "pyramidal": "depth %d; proximal %dx%d reach %d; distal 16x32 reach 6" % (d, pd, ps, pr),
        "input_active": act,
        "learning": True,
        "regrowth": False,
        "synapses_per_area": int(n_syn),
    }


def algorithmic_bytes(plan, kernel):
    """Algorithmic bytes of one launch of `kernel`, averaged over the area's
    launches of it. fused_tuft_cycle: 7 bytes per synapse (source slice, v and
    u offsets, strength and old state read; new state and flags written), 4
    per dendrite (activity read and written, raw state, state) and 12 per
    pyramidal cell-tuft (four tuft fields read, eight written)."""
    syn = sum(int(plan.layers[i].n_syns) for i in range(plan.n_layers))
    per_tuft = []
    for i in range(plan.n_layers):
        L = plan.layers[i]
        for t in range(L.n_tufts):
            T = L.tufts[t]
            n_syn = int(L.cells) * int(T.syns_per_tft)
            n_den = int(L.cells) * int(T.dens_per_tft)
            n_ct = int(L.cells) if L.kind == 2 else 0
            per_tuft.append((n_syn, n_den, n_ct))
    if kernel == "fused_tuft_cycle":
        tot = sum(7 * a + 4 * b + 12 * c for a, b, c in per_tuft)
        return tot / len(per_tuft)
    if kernel == "syn_cycle":
        return sum(4 * a for a, _, _ in per_tuft) / len(per_tuft)
    if kernel == "den_cycle_tft":
        return sum(2 * a + 4 * b for a, b, _ in per_tuft) / len(per_tuft)
    if kernel == "tft_set_syn_flags":
        return 3 * syn / plan.n_layers
    return None


class _DevBytes:
    """A u8 view of n bytes of device memory at ptr, for torch.as_tensor."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3, "strides": None, "stream": None}


def pyr_learners(flags_before, axons, prev_best_raw):
    """Pyramidal cells whose first distal tuft learns this cycle (numpy or
    torch arrays, one entry per cell): active now, CEL_PREV_ACTIVE (0x08)
    clear before the cycle, and a non-zero previous best raw state."""
    return ((flags_before & 0x08) == 0) & (axons != 0) & (prev_best_raw != 0)


def learn_syns_per_cycle(area, plan, dev_frames, flen, first, n):
    """Synapses that learning touches per cycle, counted on the device over n
    cycles (frames first .. first + n - 1 of dev_frames):
      * spiny stellate cells whose axon is non-zero after inhibition rewrite
        their tuft's synapses (ssc_mtp_simple, cl/bismit.cl:888-915);
      * pyramidal cells that became active this cycle (CEL_PREV_ACTIVE clear
        before it) and whose previous best dendrite of the first distal tuft
        had a non-zero raw state rewrite that dendrite's synapses
        (tft_dst_mtp, cl/bismit.cl:1195-1268); CEL_PREV_ACTIVE is set by the
        first distal tuft, so later ones never learn.
    Returns the mean count per cycle."""
    import torch
    from bismit_b200 import _ffi as F
    base = area.slab_ptr()
    jobs = []
    for i in range(plan.n_layers):
        L = plan.layers[i]
        ax = torch.as_tensor(_DevBytes(base + int(plan.axon_off) + int(L.axn_idz), L.cells), device="cuda")
        if L.kind == F.BM_LYR_SPINY_STELLATE and L.n_tufts:
            jobs.append(("ssc", ax, int(L.tufts[0].syns_per_tft), None, None))
        elif L.kind == F.BM_LYR_PYRAMIDAL:
            dist = [L.tufts[t] for t in range(L.n_tufts) if L.tufts[t].den_kind == F.BM_DEN_DISTAL]
            if not dist:
                continue
            T = dist[0]
            fl = torch.as_tensor(_DevBytes(base + int(L.buf_off[F.BUF["cel_flag_sets"]]), L.cells), device="cuda")
            raw = torch.as_tensor(_DevBytes(base + int(L.buf_off[F.BUF["tft_prev_best_den_states_raw"]])
                                            + int(T.cel_idz), L.cells), device="cuda")
            jobs.append(("pyr", ax, int(T.syns_per_den), fl, raw))
    total = torch.zeros((), dtype=torch.int64, device="cuda")
    for k in range(n):
        before = [j[3].clone() if j[0] == "pyr" else None for j in jobs]
        area.cycle_frames_device(dev_frames.data_ptr() + (first + k) * flen, flen, 1)
        for j, fb in zip(jobs, before):
            kind, ax, per, _, raw = j
            if kind == "ssc":
                total += (ax != 0).sum() * per
            else:
                total += pyr_learners(fb, ax, raw).sum() * per
        area.axons_touched()
    torch.cuda.synchronize()
    return int(total.item()) / n


def cycle_bytes(plan, flen, n_learn):
    """Algorithmic bytes of one cycle: 7 per synapse, 4 per dendrite, 12 per
    pyramidal cell-tuft, 4 per cell, the input frame and 3 per synapse that
    learning touches."""
    syn = sum(int(plan.layers[i].n_syns) for i in range(plan.n_layers))
    den = sum(int(plan.layers[i].n_dens) for i in range(plan.n_layers))
    ct = sum(int(plan.layers[i].n_celtfts) for i in range(plan.n_layers) if plan.layers[i].kind == 2)
    cells = sum(int(plan.layers[i].cells) for i in range(plan.n_layers))
    return 7 * syn + 4 * den + 12 * ct + 4 * cells + int(flen) + 3 * n_learn


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.p = None
        self.path = os.environ.get("BM_CLOCKS_LOG") or os.path.join("/tmp", "bm_clocks_%d_%d.csv" % (os.getpid(), gpu_index))

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                       "-i", str(self.idx), "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        mhz, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not mhz:
            return None
        return {"sm_mhz": float(np.median(mhz)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(mhz)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def live_copy_gbs(n_bytes=2 << 30, reps=5):
    """A STREAM-style device copy on this GPU (torch's copy of n_bytes, read
    plus write counted), for context beside the roofline's peak."""
    import torch
    src = torch.empty(n_bytes, dtype=torch.uint8, device="cuda")
    dst = torch.empty_like(src)
    dst.copy_(src)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    best = 0.0
    for _ in range(reps):
        e0.record()
        dst.copy_(src)
        e1.record()
        e1.synchronize()
        best = max(best, 2 * n_bytes / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del src, dst
    torch.cuda.empty_cache()
    return best


def traffic_for(kernel, workload):
    """Per-launch DRAM bytes from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        parts = line.split()
        if len(parts) >= 3 and parts[0] == kernel and parts[1] == workload:
            return float(parts[2])
    return None


def cpu_baseline(plan, slab, frames, budget_s, prefer_ref=True):
    """Times the reference kernels compiled for the CPU (oracle/_ref, all host
    threads) or, without them, the C restatement, on cycles of the same area."""
    import oracle
    kind = "reference" if (prefer_ref and oracle.load_ref() is not None) else "port"
    impl = "ref" if kind == "reference" else "port"
    threads = os.cpu_count() or 1
    work = slab.copy()
    t0 = time.perf_counter()
    n = 0
    while True:
        oracle.run(plan, work, frames[n % len(frames)][None, :], 1, start_cycle=n, threads=threads, impl=impl)
        n += 1
        if time.perf_counter() - t0 >= budget_s or n >= 1000:
            break
    dt = time.perf_counter() - t0
    return {"value": int(plan.n_syns_total) * n / dt, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": "%d cycle(s) of %s on the host cores (%.1f s)" % (n, "the same area", dt)}


def measure_parity(area, plan, frames, n):
    """Cycles the area n times through the public API with host frames and
    compares its whole state slab (every axon, synapse, dendrite, tuft and
    cell byte) with bismit's own kernels compiled for the CPU (oracle/_ref;
    the C restatement when that was not built) run from the same state on the
    same frames."""
    import oracle
    impl = "ref" if oracle.load_ref() is not None else "port"
    ref = area.read_slab()
    c0 = area.cycle_count()
    for k in range(n):
        area.write_input(frames[k])
        area.cycle(1)
    dev = area.read_slab()
    t0 = time.perf_counter()
    oracle.run(plan, ref, frames[:n], n, start_cycle=c0, threads=os.cpu_count() or 1, impl=impl)
    t_ora = time.perf_counter() - t0
    diff = int(np.count_nonzero(dev != ref))
    return {"identical": diff == 0, "differing_bytes": diff, "bytes_compared": int(ref.size), "cycles": n,
            "from_cycle": int(c0), "learning": True,
            "against": ("bismit's cl/*.cl compiled for the CPU (oracle/_ref)" if impl == "ref"
                        else "the C restatement of bismit's kernels (oracle)"),
            "what": "whole state slab after each run: axons, synapse states, strengths, sources and flags, "
                    "dendrite, tuft and cell buffers",
            "oracle_s": round(t_ora, 2)}


SOAK_S = 0.6   # seconds of the same cycles on each side of a timed region, for the clock samples


def soak(fn, stream, seconds):
    """Keeps the GPU on the timed workload for `seconds` (nvidia-smi samples
    every 200 ms, longer than most timed regions)."""
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        fn()
        stream.synchronize()


def alg_bytes_cycle(plan):
    """Algorithmic bytes of one full cycle: 7 per synapse, 4 per dendrite, 12
    per cell-tuft, 4 per cell, plus the input frame."""
    b = 0
    for i in range(plan.n_layers):
        L = plan.layers[i]
        b += 7 * int(L.n_syns) + 4 * int(L.n_dens) + 4 * int(L.cells)
        if L.kind == 2:
            b += 12 * int(L.cells) * int(L.n_tufts)
    if plan.n_inputs:
        b += int(plan.inputs[0].len)
    return b


def batch_profile(batch, frames, fb, W, K):
    """Per-step device time of K eager cycles of a batch (CUDA events on its
    stream, graph bypassed): {step: [areas, ms per cycle]}."""
    batch.reset_profile()
    batch.set_profiling(True)
    batch.cycle_frames_device(frames.data_ptr() + W * fb, K)
    prof = batch.profile()
    batch.set_profiling(False)
    return {"%s L%d.%d" % (n, l, i): [a, round(ms / K, 4)] for (n, l, i, a, _c, ms) in prof}


def slabs_equal(arms):
    """Whether every arm's areas hold the same whole state slabs (arms: lists
    of areas in the same order), read one area at a time."""
    for group in zip(*arms):
        first = group[0].read_slab()
        if not all(np.array_equal(first, a.read_slab()) for a in group[1:]):
            return False
    return True


def run_batched(args, ctx, stream, K, W, ws):
    """The batched-instances workload: `--batch-instances` independent areas of
    uneven size (configs.batch_instances), cycled on the same seeded frames
    (a) as one batch with graph replay, (b) one area after another with the
    same fused kernels (one launch sequence per area, no graph), and (c) in
    the plain form, one area after another with one kernel per reference
    stage. (a) against (b) isolates batching and graph replay; (b) against
    (c) is the fusion. The three arms' whole state slabs are compared after
    the same cycles. Returns the JSON object."""
    import torch
    from bismit_b200 import configs, cortex, map as M
    n = args.batch_instances
    ins = configs.batch_instances(n, args.seed)
    areas_b, areas_f, areas_p, frames_h = [], [], [], []
    for i, (side, depth, dens, syns, act) in enumerate(ins):
        lmaps, areas = configs.instance_area(side, depth, dens, syns)
        seed = args.seed * 1000 + i
        areas_b.append(cortex.CorticalArea(ctx, M.area_desc("v1", lmaps, areas, configs.bench_settings()), seed))
        areas_f.append(cortex.CorticalArea(ctx, M.area_desc("v1", lmaps, areas, configs.bench_settings()), seed))
        areas_p.append(cortex.CorticalArea(ctx, M.area_desc("v1", lmaps, areas,
                                                            configs.bench_settings().plain_kernels()), seed))
        frames_h.append(configs.frames(K + W, areas_b[-1].input_len(), act, seed))
    n_syn = sum(int(a.plan.n_syns_total) for a in areas_b)
    alg = sum(alg_bytes_cycle(a.plan) for a in areas_b)
    batch = cortex.Batch(ctx, areas_b)
    t_tune = time.perf_counter()
    tuned = batch.autotune(None)
    t_tune = time.perf_counter() - t_tune
    fb = batch.frame_bytes()
    packed = torch.from_numpy(batch.pack_frames(frames_h)).to("cuda")
    per_area = [torch.from_numpy(f).to("cuda") for f in frames_h]
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    from bismit_b200.replicas import max_over_ranks

    def max_ms(ms):
        return max_over_ranks(ms, "cuda")

    def timed(fn):
        fn(0, W)
        torch.cuda.synchronize()
        e0.record(stream)
        fn(W, K)
        e1.record(stream)
        torch.cuda.synchronize()
        return max_ms(e0.elapsed_time(e1))

    def batched_cycles(c0, nc):
        batch.cycle_frames_device(packed.data_ptr() + c0 * fb, nc)

    def one_by_one(arm):
        def run(c0, nc):
            for c in range(c0, c0 + nc):
                for a, f in zip(arm, per_area):
                    a.cycle_frames_device(f.data_ptr() + c * f.shape[1], f.shape[1], 1)
        return run

    ms_b = timed(batched_cycles)
    ms_f = timed(one_by_one(areas_f))
    ms_p = timed(one_by_one(areas_p))
    same = slabs_equal([areas_b, areas_f, areas_p])
    steps_b = batch_profile(batch, packed, fb, W, K)
    peak, peak_kind = peaks()

    def arm(ms, launches, **kw):
        d = {"value": n_syn * K * ws / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / K, "launches_per_cycle": launches,
             "hbm_frac": round(alg / (ms / K / 1e3) / 1e9 / peak, 4)}
        d.update(kw)
        return d

    out = {
        "workload": "batch_%d" % n, "instances": n, "synapses": n_syn,
        "sizes": "side 32..192 step 16, depth 1..4, distal dens {8,16} x syns {16,32,64}, proximal 1x1, "
                 "spiny stellate 1x32; active 1-4%",
        "batched": arm(ms_b, batch.launches_per_cycle(), graph=True, algorithmic_bytes_per_cycle=alg,
                       autotuned_steps=tuned, autotune_s=round(t_tune, 2)),
        "fused_single": arm(ms_f, sum(a.launches_per_cycle() for a in areas_f), graph=False),
        "plain": arm(ms_p, sum(a.launches_per_cycle() for a in areas_p), graph=False),
        "batched_over_fused_single": round(ms_f / ms_b, 3),
        "batched_over_plain": round(ms_p / ms_b, 3),
        "slabs_identical": bool(same),
        "compared": "whole state slab of every instance, three arms, after %d cycles" % (W + K),
        "steps": steps_b,
        "peak_source": peak_kind,
    }
    batch.close()
    for a in areas_b + areas_f + areas_p:
        a.close()
    return out


def run_hierarchy(args, ctx, stream, K, W, ws):
    """The three-area hierarchy (128 -> 192 -> 96, depth 2, feed-forward and
    feedback tracts, input 2 % active), on the same seeded frames: (a) one
    batch with its tracts, replayed from a CUDA graph; (b) the same fused
    kernels one area after another (one launch sequence per area, no graph)
    and (c) the plain form, one kernel per reference stage, one area after
    another. (b) and (c) deliver the tracts as the batch does: at the head of
    each cycle every tract copies its source's output of the previous cycle
    (bm_area_deliver_tract), then the areas cycle. The three arms' whole state slabs are compared."""
    import torch
    from bismit_b200 import Cortex, configs, cortex, map as M
    lmaps, areas, names = configs.hierarchy()
    cx = Cortex(lmaps, areas, configs.bench_settings(), seed=args.seed, ctx=ctx)
    batched = [cx.area(n) for n in names]
    single = [cortex.CorticalArea(ctx, M.area_desc(n, lmaps, areas, configs.bench_settings()), args.seed)
              for n in names]
    plain = [cortex.CorticalArea(ctx, M.area_desc(n, lmaps, areas, configs.bench_settings().plain_kernels()),
                                 args.seed) for n in names]
    fb = cx.batch.frame_bytes()
    fr = torch.from_numpy(configs.frames(K + W, fb, 0.02, args.seed + 3)).to("cuda")
    n_syn = sum(int(a.plan.n_syns_total) for a in batched)
    alg = sum(alg_bytes_cycle(a.plan) for a in batched)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    from bismit_b200.replicas import max_over_ranks

    def max_ms(ms):
        return max_over_ranks(ms, "cuda")

    def timed(fn):
        fn(0, W)
        torch.cuda.synchronize()
        e0.record(stream)
        fn(W, K)
        e1.record(stream)
        torch.cuda.synchronize()
        return max_ms(e0.elapsed_time(e1))

    t_tune = time.perf_counter()
    tuned = cx.batch.autotune(None)
    t_tune = time.perf_counter() - t_tune

    def batched_cycles(c0, nc):
        cx.batch.cycle_frames_device(fr.data_ptr() + c0 * fb, nc)

    def one_by_one(arm):
        def run(c0, nc):
            for c in range(c0, c0 + nc):
                for (sk, so, dk, di, off, _n) in cx.tracts:
                    arm[dk].deliver_tract(arm[sk], so, di, off)
                arm[0].cycle_frames_device(fr.data_ptr() + c * fb, fb, 1)
                for a in arm[1:]:
                    a.cycle(1)
        return run

    ms_b = timed(batched_cycles)
    ms_f = timed(one_by_one(single))
    ms_p = timed(one_by_one(plain))
    same = slabs_equal([batched, single, plain])
    peak, _ = peaks()
    steps_h = batch_profile(cx.batch, fr, fb, W, K)

    def arm(ms, launches, **kw):
        d = {"value": n_syn * K * ws / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / K, "launches_per_cycle": launches,
             "hbm_frac": round(alg / (ms / K / 1e3) / 1e9 / peak, 4)}
        d.update(kw)
        return d

    out = {
        "steps": steps_h,
        "workload": "hierarchy_3", "areas": "128x128 -> 192x192 -> 96x96, depth 2", "synapses": n_syn,
        "tracts": len(cx.tracts),
        "batched": arm(ms_b, cx.batch.launches_per_cycle(), graph=True, autotuned_steps=tuned,
                       autotune_s=round(t_tune, 2)),
        "fused_single": arm(ms_f, sum(a.launches_per_cycle() for a in single) + len(cx.tracts), graph=False),
        "plain": arm(ms_p, sum(a.launches_per_cycle() for a in plain) + len(cx.tracts), graph=False),
        "batched_over_fused_single": round(ms_f / ms_b, 3),
        "batched_over_plain": round(ms_p / ms_b, 3),
        "slabs_identical": bool(same),
        "compared": "whole state slab of every area, three arms, after %d cycles" % (W + K),
    }
    if ws == 1 and not args.no_cpu_baseline:
        plans = [a.plan for a in batched]
        slabs = [a.read_slab() for a in batched]
        tracts, _ext = M.area_tracts(lmaps, areas, names, plans)
        out["cpu_baseline"] = hierarchy_cpu_baseline(plans, slabs, tracts, args.cpu_sample_seconds / 2, args.seed)
    for a in single + plain:
        a.close()
    cx.close()
    return out


def hierarchy_cpu_baseline(plans, slabs, tracts, budget_s, seed):
    """bismit's kernels compiled for the CPU (oracle/_ref, all host threads;
    the C restatement without it) on cycles of the hierarchy, each area after
    its tract intakes (previous-cycle outputs) as on the device."""
    import oracle
    impl = "ref" if oracle.load_ref() is not None else "port"
    threads = os.cpu_count() or 1
    from bismit_b200 import configs
    ext = configs.frames(8, int(plans[0].inputs[0].len), 0.02, seed + 5)
    n_syn = sum(int(p.n_syns_total) for p in plans)
    t0 = time.perf_counter()
    n = 0
    while True:
        outs = [sl[int(p.axon_off):].copy() for p, sl in zip(plans, slabs)]
        for (si, o, d, i, off, ln) in tracts:
            src = int(plans[si].outputs[o].axn_idz)
            oracle.intake(plans[d], slabs[d], i, off, outs[si][src:src + ln])
        oracle.intake(plans[0], slabs[0], 0, 0, ext[n % len(ext)])
        for p, sl in zip(plans, slabs):
            oracle.run(p, sl, None, 1, start_cycle=n, threads=threads, impl=impl)
        n += 1
        if time.perf_counter() - t0 >= budget_s or n >= 1000:
            break
    dt = time.perf_counter() - t0
    return {"value": n_syn * n / dt, "unit": UNIT, "cores": threads,
            "kind": "reference" if impl == "ref" else "port",
            "sample": "%d cycle(s) of the three areas with their tract intakes (%.1f s)" % (n, dt)}


def run_small_area(args, ctx, stream, n_cycles=1000):
    """area_64 (64 x 64 columns, 2.23 M synapses; its 16 MB per cycle stay in
    L2, so it is judged on cycles/s): n_cycles cycles over device frames timed
    with CUDA events, beside bismit's kernels compiled for the CPU on the same
    area and frames (bounded sample)."""
    import torch
    from bismit_b200 import configs, cortex, map as M
    lmaps, areas, act = configs.workload("area_64")
    area = cortex.CorticalArea(ctx, M.area_desc("v1", lmaps, areas, configs.bench_settings()), args.seed + 64)
    plan = area.plan
    flen = area.input_len()
    warm = 10
    fr = configs.frames(n_cycles + warm, flen, act, args.seed + 64)
    init = area.read_slab()
    dev = torch.from_numpy(fr).to("cuda")
    area.cycle_frames_device(dev.data_ptr(), flen, warm)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    area.cycle_frames_device(dev.data_ptr() + warm * flen, flen, n_cycles)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    n_syn = int(plan.n_syns_total)
    out = {"workload": "area_64", "columns": "64x64", "synapses": n_syn, "cycles": n_cycles,
           "value": n_syn * n_cycles / (ms / 1e3), "unit": UNIT, "cycles_per_s": round(n_cycles / (ms / 1e3), 1),
           "ms_per_step": ms / n_cycles, "launches_per_cycle": area.launches_per_cycle()}
    # The same area as a batch of one, its cycle replayed from a CUDA graph
    # (same seed and frames, so the two end states must be equal).
    twin = cortex.CorticalArea(ctx, M.area_desc("v1", lmaps, areas, configs.bench_settings()), args.seed + 64)
    b = cortex.Batch(ctx, [twin])
    b.cycle_frames_device(dev.data_ptr(), warm)
    torch.cuda.synchronize()
    e0.record(stream)
    b.cycle_frames_device(dev.data_ptr() + warm * flen, n_cycles)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_g = e0.elapsed_time(e1)
    out["graph"] = {"value": n_syn * n_cycles / (ms_g / 1e3), "unit": UNIT,
                    "cycles_per_s": round(n_cycles / (ms_g / 1e3), 1), "ms_per_step": ms_g / n_cycles,
                    "launches_per_cycle": b.launches_per_cycle(),
                    "states_identical": bool(np.array_equal(area.read_slab(), twin.read_slab()))}
    b.close()
    twin.close()
    area.close()
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(plan, init, fr[warm:], args.cpu_sample_seconds / 2)
    return out


def run_serving(args, ctx):
    """Serving: sessions drawn from the batched workload's size distribution
    arrive as a Poisson process (--serve-rate per second), each streaming
    100-2000 seeded frames (cycled from a pool of 8 per session), admitted by a
    device-memory budget (--serve-budget-gb) and batched tick by tick.
    Returns the JSON object with p50/p99 per-frame latency."""
    from bismit_b200 import configs, cortex, map as M, plan_of
    n = args.serve_sessions
    rng = np.random.default_rng([args.seed, 0x73657276])
    ins = configs.batch_instances(n, args.seed + 7)
    arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, n))
    n_frames = rng.integers(100, 2001, n)
    descs, pools = [], []
    for i, (side, depth, dens, syns, act) in enumerate(ins):
        lmaps, areas = configs.instance_area(side, depth, dens, syns)
        d = M.area_desc("v1", lmaps, areas, configs.bench_settings())
        descs.append(d)
        pools.append(configs.frames(8, side * side, act, args.seed * 7919 + i))
    srv = cortex.Server(ctx, int(args.serve_budget_gb * 1e9))
    opened, total, queued = 0, 0, 0
    t_tick = t_submit = 0.0
    tick_calls = []
    t0 = time.perf_counter()
    while True:
        now = time.perf_counter() - t0
        while opened < n and arrivals[opened] <= now:
            ts = time.perf_counter()
            sid = srv.open(descs[opened], args.seed * 1000 + opened)
            k = int(n_frames[opened])
            for r in range(k // 8):
                srv.submit(sid, pools[opened])
            if k % 8:
                srv.submit(sid, pools[opened][:k % 8])
            t_submit += time.perf_counter() - ts
            srv.close_session(sid)
            total += k
            opened += 1
        ts = time.perf_counter()
        cycled = srv.tick()
        dt = time.perf_counter() - ts
        t_tick += dt
        tick_calls.append(dt)
        queued += cycled
        if opened == n and queued >= total:
            srv.drain()
            break
        if cycled == 0 and opened < n:
            time.sleep(max(0.0, min(0.001, arrivals[opened] - (time.perf_counter() - t0))))
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    return {
        "workload": "serving_%d" % n, "sessions": n, "arrival_rate_per_s": args.serve_rate,
        "frames_per_session": "uniform 100..2000", "frames": int(st["frames"]),
        "sizes": "as the batched workload (side 32..192, depth 1..4, distal {8,16} x {16,32,64})",
        "budget_bytes": int(st["budget_bytes"]),
        "value": st["syn_cycles"] / st["span_s"] if st["span_s"] else None, "unit": UNIT,
        "p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3), "mean_ms": round(st["mean_ms"], 3),
        "ticks": int(st["ticks"]), "batch_rebuilds": int(st["batch_rebuilds"]),
        "rebuild_s": round(st["rebuild_s"], 3), "rebuild_drains": st["rebuild_drains"],
        "capture_s": round(st["capture_s"], 3), "admit_s": round(st["admit_s"], 3), "gpu_s": round(st["gpu_s"], 3),
        "tick_device_p99_ms": round(st["tick_p99_ms"], 3), "tick_device_max_ms": round(st["tick_max_ms"], 3),
        "tick_device_max_at": {"tick": int(st["tick_max_no"]), "sessions": int(st["tick_max_members"]),
                               "with": [w for w, b in (("first", 1), ("rebuild", 2), ("drain", 4), ("capture", 8))
                                        if int(st["tick_max_what"]) & b],
                               "queue_ms": round(st["tick_max_queue_ms"], 3),
                               "builder": [w for w, b in (("build", 1), ("batch_free", 2), ("buffer_free", 4),
                                                          ("area_free", 8), ("output_free", 16))
                                           if int(st["tick_max_builder"]) & b],
                               "builder_longest_ms": round(st["tick_max_builder_ms"], 3)},
        "tick_call_slowest": [[int(i), round(tick_calls[i] * 1e3, 3)] for i in np.argsort(tick_calls)[-3:][::-1]]
        if tick_calls else None,
        "tick_call_p99_ms": round(float(np.percentile(tick_calls, 99)) * 1e3, 3) if tick_calls else None,
        "tick_call_max_ms": round(max(tick_calls) * 1e3, 3) if tick_calls else None,
        "tick_call_s": round(t_tick, 3), "submit_s": round(t_submit, 3), "wall_s": round(wall, 3),
        "latency": "per frame: tick completion minus the moment the frame was ready (its session's previous "
                   "frame done, or its arrival); admission waits included",
    }


def run_ours(args):
    import torch
    from bismit_b200 import configs, cortex, map as M

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    lmaps, areas, act = configs.workload(args.workload)
    st = configs.bench_settings()
    if args.path == "plain":
        st.plain_kernels()
    desc = M.area_desc("v1", lmaps, areas, st)
    ctx = cortex._Ctx(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    from bismit_b200.replicas import frame_seed, max_over_ranks, replica_seed
    area = cortex.CorticalArea(ctx, desc, seed=replica_seed(args.seed, rank))
    plan = area.plan
    flen = area.input_len()
    K, W = args.steps, args.warmup
    nfr = K + W
    host_frames = configs.frames(nfr, flen, act, frame_seed(args.seed, rank))
    dev_frames = torch.from_numpy(host_frames).to("cuda")

    def barrier():
        if ws > 1:
            torch.distributed.barrier()

    init_slab = area.read_slab() if (rank == 0 and ws == 1 and not args.no_cpu_baseline) else None
    out_len = area.output_len()
    # Bit-exactness at this size, measured: a few cycles through the public
    # API against bismit's kernels on the host (untimed; the timed cycles
    # continue from the state they leave).
    parity = measure_parity(area, plan, host_frames, args.parity_cycles) if (rank == 0 and args.parity_cycles) else None

    # warm-up
    area.cycle_frames_device(dev_frames.data_ptr(), flen, W)
    torch.cuda.synchronize()
    barrier()
    clocks = Clocks(local)
    clocks.start()
    soak(lambda: area.cycle_frames_device(dev_frames.data_ptr(), flen, W), stream, SOAK_S)
    torch.cuda.synchronize()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    area.cycle_frames_device(dev_frames.data_ptr() + W * flen, flen, K)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    soak(lambda: area.cycle_frames_device(dev_frames.data_ptr(), flen, W), stream, SOAK_S)
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), "cuda")
    # The cycle's kernels plus each cycle's frame intake (one copy kernel).
    launches = (area.launches_per_cycle() + 1) * K
    n_syn = int(plan.n_syns_total)
    value = n_syn * K * ws / (ms / 1e3)

    # Per-kernel times (library CUDA events on this stream) for the roofline.
    area.reset_profile()
    area.set_profiling(True)
    area.cycle_frames_device(dev_frames.data_ptr() + W * flen, flen, K)
    torch.cuda.synchronize()
    prof = area.profile()
    area.set_profiling(False)
    dom = max(prof.items(), key=lambda kv: kv[1][1])
    dom_name, (dom_launches, dom_ms) = dom
    avg_ms = dom_ms / dom_launches
    alg = algorithmic_bytes(plan, dom_name)
    peak, peak_kind = peaks()
    copy_live = live_copy_gbs()
    roofline = None
    if alg is not None:
        ach = alg / (avg_ms / 1e3) / 1e9
        tr = traffic_for(dom_name, args.workload)
        roofline = {"bound": "hbm", "kernel": dom_name, "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                    "frac": round(ach / peak, 4), "peak_source": peak_kind, "traffic": tr,
                    "algorithmic_bytes_per_launch": int(alg), "avg_launch_ms": round(avg_ms, 4),
                    "share": round(dom_ms / sum(v[1] for v in prof.values()), 3),
                    "live_copy_gbs": round(copy_live, 1), "frac_of_live_copy": round(ach / copy_live, 4)}

    # The whole cycle against the same peak: algorithmic bytes per cycle with
    # the synapses that learning touches counted on the device (untimed
    # cycles of the same frames), over the timed cycle time.
    n_count = min(K, 20)
    n_learn = learn_syns_per_cycle(area, plan, dev_frames, flen, W, n_count)
    b_cycle = cycle_bytes(plan, flen, n_learn)
    cyc_gbs = b_cycle / (ms / K / 1e3) / 1e9
    cycle_roofline = {"bytes_per_cycle": int(b_cycle), "learn_syns_per_cycle": round(n_learn, 1),
                      "learn_counted_over_cycles": n_count, "achieved": round(cyc_gbs, 1), "peak": peak,
                      "unit": "GB/s", "frac": round(cyc_gbs / peak, 4), "peak_source": peak_kind,
                      "frac_of_live_copy": round(cyc_gbs / copy_live, 4)}

    # End to end through the public API with host buffers: each cycle's frame
    # goes in with bm_area_write_input from pinned host memory, and each
    # cycle's output axons come back through a sampler with backpressure
    # (CorticalArea::sampler, the reference's per-cycle readback), taken by a
    # receiver thread as a sampler's TractReceiver is. Backpressure makes every
    # cycle's frame arrive (none skipped); the cycling thread enqueues the next
    # cycle while the receiver waits for the previous frame. The same receiver
    # thread takes the W warm-up cycles' frames first, so its start-up is not
    # timed.
    import ctypes
    import threading
    pin_in = torch.from_numpy(host_frames).pin_memory()
    pin_out = torch.empty(out_len, dtype=torch.uint8).pin_memory()
    lib = area.lib
    # The output's layer_idx indexes the layer map; the sampler takes the
    # data (cellular) layer that owns those slices.
    out_layer = area.data_layer(area.layer_names[int(plan.outputs[0].layer_idx)])
    smp = area.sampler("axons", out_layer, backpressure=True)
    if smp.len != out_len:
        raise RuntimeError("output sampler covers %d bytes, the output slice %d" % (smp.len, out_len))
    smp.set_timeout(60000)
    got_cycles = []
    recv_err = []
    t_recv = []     # host time each frame was taken
    t_call = []     # host time of each cycle's write_input + cycle calls

    def receive():
        cyc, got = ctypes.c_uint64(), ctypes.c_int()
        for _ in range(W + K):
            rc = lib.bm_sampler_recv(smp.h, 1, ctypes.c_void_p(pin_out.data_ptr()), ctypes.c_uint64(out_len),
                                     ctypes.byref(cyc), ctypes.byref(got))
            if rc != 0 or not got.value:
                recv_err.append(rc)
                return
            t_recv.append(time.perf_counter())
            got_cycles.append(cyc.value)

    def host_cycles(k0, n):
        for k in range(k0, k0 + n):
            ta = time.perf_counter()
            if lib.bm_area_write_input(area.h, 0, ctypes.c_void_p(pin_in[k].data_ptr()), ctypes.c_size_t(flen)):
                raise RuntimeError("bm_area_write_input failed")
            if lib.bm_area_cycle(area.h, 1):
                raise RuntimeError("bm_area_cycle failed")
            t_call.append(time.perf_counter() - ta)

    rx = threading.Thread(target=receive)
    rx.start()
    host_cycles(0, W)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    e0.record(stream)
    host_cycles(W, K)
    e1.record(stream)
    rx.join()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_wall = time.perf_counter() - t0
    smp.close()
    if recv_err or len(got_cycles) != W + K or got_cycles != list(range(got_cycles[0], got_cycles[0] + W + K)):
        raise RuntimeError("output sampler: %d of %d cycles received in order" % (len(got_cycles), W + K))
    barrier()
    e2e_ms = max_over_ranks(e2e_ms, "cuda")
    e2e_val = n_syn * K * ws / (e2e_ms / 1e3)
    # Host-side view of the timed cycles: each cycle's calls, the gaps between
    # frames reaching the receiver, and the wall time to the last frame.
    calls = np.array(t_call[W:]) * 1e3
    gaps = np.diff(np.array(t_recv[W - 1:])) * 1e3 if W > 0 else np.diff(np.array(t_recv)) * 1e3
    e2e_host = {"call_ms_median": round(float(np.median(calls)), 4), "call_ms_max": round(float(calls.max()), 4),
                "frame_gap_ms_median": round(float(np.median(gaps)), 4), "frame_gap_ms_max": round(float(gaps.max()), 4),
                "wall_ms_to_last_frame": round((t_recv[-1] - t0) * 1e3, 3), "device_ms": round(e2e_ms, 3)}

    area.close()
    batched = None if args.no_batched else run_batched(args, ctx, stream, K, W, ws)
    hierarchy = None if args.no_hierarchy else run_hierarchy(args, ctx, stream, K, W, ws)
    serving = None if (args.no_serving or ws > 1) else run_serving(args, ctx)
    small = None if (args.no_small or ws > 1) else run_small_area(args, ctx, stream)

    cpu = None
    if init_slab is not None:
        cpu = cpu_baseline(plan, init_slab, host_frames, args.cpu_sample_seconds)

    if rank == 0:
        cfg = workload_config(args.workload, n_syn)
        setup = {"path": args.path, "areas": ws, "parallelism": "replicas x%d" % ws,
                 "l2": "state slab %.2f GB per area > 126 MB L2, no flush needed" % (plan.slab_bytes / 1e9),
                 "clocks_window": "nvidia-smi every 200 ms over the timed region plus %.1f s of the same "
                                  "cycles on each side" % SOAK_S}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8/i8", "data": "synthetic (seeded frames, seeded synapse growth)", "config": cfg,
            "setup": setup, "clocks": clk,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": flen, "d2h_bytes_per_step": out_len,
                    "wall_s": round(e2e_wall, 4), "host": e2e_host},
            "gpu_launches": launches,
            "roofline": roofline,
            "cycle_roofline": cycle_roofline,
            "cpu_baseline": cpu,
            "parity": parity,
            "kernels": {k: {"launches": v[0], "ms": round(v[1], 4)} for k, v in prof.items()},
            "batched_instances": batched,
            "hierarchy": hierarchy,
            "serving": serving,
            "small_area": small,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


def run_profile(args):
    """A short, fixed launch sequence for a profiler: W warm-up cycles, then K
    cycles between CUDA events, of one workload on cuda:0; prints one JSON
    line with the device time (informational: a run under a profiler is no
    bench value). Area cycles are plain launches; the batch replays its CUDA
    graph (under `--profile-run batched` its launch list is the graph's
    kernels)."""
    import torch
    from bismit_b200 import configs, cortex, map as M
    torch.cuda.set_device(0)
    ctx = cortex._Ctx(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    K, W = args.steps, args.warmup
    areas = []
    if args.profile_run == "area":
        if args.workload == "smoother":
            (lmaps, ar), act = configs.smoother_area(), 0.03
        elif args.workload == "retina":
            (lmaps, ar), act = configs.retina_area(48, n_filters=2, src_depth=2), 0.05
        else:
            lmaps, ar, act = configs.workload(args.workload)
        st = M.CorticalAreaSettings().strengths_start_at_zero() if args.regrowth else configs.bench_settings()
        if args.path == "plain":
            st.plain_kernels()
        areas.append(cortex.CorticalArea(ctx, M.area_desc("v1", lmaps, ar, st), seed=args.seed + 1))
        flen = areas[0].input_len()
        dev = torch.from_numpy(configs.frames(K + W, flen, act, args.seed)).to("cuda")

        def cycles(c0, n):
            areas[0].cycle_frames_device(dev.data_ptr() + c0 * flen, flen, n)
        launches = areas[0].launches_per_cycle
        name = args.workload + (" with regrowth" if args.regrowth else "")
    elif args.profile_run == "encoders":
        from bismit_b200 import encode as E
        n, side = 64, 256
        frames = torch.zeros(n, side * side, dtype=torch.uint8, device="cuda")
        images = torch.randint(0, 256, (n, 28, 28), dtype=torch.uint8, device="cuda")
        vals = np.linspace(0.0, 0.95, n, dtype=np.float32)   # the SDR writer takes values below the top
        sdr = E.ScalarSdrWriter(ctx, (0.0, 1.0), 0.05, (side, side), seed=args.seed)

        def cycles(c0, k):
            for _ in range(k):
                E.encode_2d_image(ctx, images, (28, 28), (side, side), 1.0, frames)
                E.encode_scalar(ctx, vals, (0.0, 1.0), (side, side), frames, seed=args.seed)
                E.encode_scalar_glyph(ctx, vals, (0.0, 1.0), (side, side), frames)
                sdr.encode(vals, frames)
                E.encode_hex_mold_scaled(ctx, 6, (side, side), (side, side), frames[0])
        launches = lambda: 5
        name = "encoders: 64 frames of 256 x 256 per encoder"
    elif args.profile_run == "hierarchy":
        from bismit_b200 import Cortex
        lmaps, ar, names = configs.hierarchy()
        cx = Cortex(lmaps, ar, configs.bench_settings(), seed=args.seed, ctx=ctx)
        batch = cx.batch
        batch.autotune(args.autotune_cache)
        fb = batch.frame_bytes()
        dev = torch.from_numpy(configs.frames(K + W, fb, 0.02, args.seed + 3)).to("cuda")
        hier_syn = sum(int(cx.area(n).plan.n_syns_total) for n in names)

        def cycles(c0, n):
            batch.cycle_frames_device(dev.data_ptr() + c0 * fb, n)
        launches = batch.launches_per_cycle
        name = "hierarchy_3"
    else:
        frames_h = []
        for i, (side, depth, dens, syns, act) in enumerate(configs.batch_instances(args.batch_instances, args.seed)):
            lmaps, ar = configs.instance_area(side, depth, dens, syns)
            seed = args.seed * 1000 + i
            areas.append(cortex.CorticalArea(ctx, M.area_desc("v1", lmaps, ar, configs.bench_settings()), seed))
            frames_h.append(configs.frames(K + W, areas[-1].input_len(), act, seed))
        batch = cortex.Batch(ctx, areas)
        batch.autotune(args.autotune_cache)
        fb = batch.frame_bytes()
        dev = torch.from_numpy(batch.pack_frames(frames_h)).to("cuda")

        def cycles(c0, n):
            batch.cycle_frames_device(dev.data_ptr() + c0 * fb, n)
        launches = batch.launches_per_cycle
        name = "batch_%d" % args.batch_instances
    torch.cuda.synchronize()
    cycles(0, W)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    cycles(W, K)
    e1.record(stream)
    torch.cuda.synchronize()
    n_syn = hier_syn if args.profile_run == "hierarchy" else sum(int(a.plan.n_syns_total) for a in areas)
    if args.profile_run == "encoders":
        sdr.close()
    print(json.dumps({"profile_run": name, "steps": K, "warmup": W, "launches_per_cycle": launches(),
                      "synapses": n_syn, "ms_per_cycle": e0.elapsed_time(e1) / K}), flush=True)
    if args.profile_run == "batched":
        batch.close()
    if args.profile_run == "hierarchy":
        cx.close()
    for a in areas:
        a.close()
    ctx.close()


def run_reference(args):
    """The reference's own kernels (cl/*.cl compiled for the CPU, all host
    threads) on the same workload; rank 0 only."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    import oracle
    from oracle import plan as OP
    from bismit_b200 import configs, map as M
    if oracle.load_ref() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (bismit's cl/*.cl compiled for the CPU) "
                                                             "was not built: no bismit checkout at build time"}))
        return
    lmaps, areas, act = configs.workload(args.workload)
    desc = M.area_desc("v1", lmaps, areas, configs.bench_settings())
    # The oracle's own restatement of bismit's map code: this arm loads none
    # of the library's native code.
    plan = OP.resolve(desc, args.seed + 1)
    slab = np.zeros(int(plan.slab_bytes), np.uint8)
    oracle.grow(plan, slab, args.seed + 1, desc.init_flags)
    flen = int(plan.inputs[0].len)
    fr = configs.frames(args.steps + args.warmup, flen, act, args.seed)
    threads = os.cpu_count() or 1
    for k in range(args.warmup):
        oracle.run(plan, slab, fr[k][None, :], 1, start_cycle=k, threads=threads, impl="ref")
    t0 = time.perf_counter()
    for k in range(args.steps):
        oracle.run(plan, slab, fr[args.warmup + k][None, :], 1, start_cycle=args.warmup + k, threads=threads, impl="ref")
    dt = time.perf_counter() - t0
    value = int(plan.n_syns_total) * args.steps / dt
    cfg = workload_config(args.workload, plan.n_syns_total)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8/i8", "data": "synthetic (seeded frames, seeded synapse growth)", "config": cfg,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": "%d full cycles of the area" % args.steps},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.profile_run:
        run_profile(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
