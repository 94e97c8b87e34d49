// bm_batch.cu -- batched cycling: several areas (instances of uneven column
// grids that share one layer map and settings) advanced together, one launch
// per stage step for all of them, the whole cycle replayed from a CUDA graph.
//
// Every area keeps its own state slab, control block and slice table; a batch
// only adds per-step job tables in device memory. Each step of the common stage
// program (bm_area.h) becomes:
//   * tuft steps: one k_fused_tuft_batch launch over every area's tiles when
//     all of them are tiled and share a ring geometry, else each area's own
//     launches;
//   * per-cell steps (soma, inhibition, outputs, learning): one launch whose
//     blocks are split among the areas by a block prefix table, running the
//     same per-item bodies as the one-area kernels (bm_items.cuh);
//   * cycle end: one launch advancing every area's device cycle counter.
// Inputs come from tracts (another area's output axons, bm_batch_connect),
// from each area's own bm_area_write_input, or for
// bm_batch_cycle_frames_device from a device array of per-cycle frame blocks.
// One copy launch at the head of each cycle does the tracts and the frame
// intake, so every tract carries its source's output of the previous cycle.
//
// A project-written autotuner (bm_batch_autotune) picks, for each batched
// tuft step, the tile size, the ring's depth and the resident CTAs per SM by
// timing candidates on the live batch (with the touched buffers saved and
// restored), and can keep its choices in a cache file.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "bm_area.h"
#include "bm_items.cuh"

using namespace bm;

namespace {

// One area's share of a batched per-cell step.
struct CellJob {
    DevLayer L;
    uint8_t* axns;
    const SliceRec* slices;
    AreaCtl* ctl;
    uint64_t key;       // inhibition rnd key (other steps take theirs from L)
    int32_t radius;     // inhibition radius
    int32_t ctrl;       // pyramidal tail: 0 none, 1 intra-column, 2 output
    uint32_t learn;     // fused steps: learning included
    uint32_t x;         // tuft or control index
    uint32_t tufts;     // pyramidal tail: per-cell tufts folded in (bit t)
    uint32_t n;         // work items (cells or columns)
    uint32_t block0;    // first block of this job
};

// One copy at the head of a cycle: a tract (src is a device pointer) or an
// input taken from the cycle's frame block (src_off within the block).
struct IntakeJob {
    uint8_t* dst;
    const uint8_t* src;  // tract source, or null: from the frame block
    uint64_t src_off;
    uint32_t len;
    uint32_t block0;
};

struct BatchCtl {
    const uint8_t* frames;   // per-cycle frame blocks, or null (inputs written per area)
    uint64_t cursor;         // cycles done since the current call began
    uint64_t frame_bytes;    // bytes of one cycle's block
};

// An unfused tuft's four stages, one thread per cell (tuft_cell_item).
constexpr int BK_TUFT_CELLS = 100;

constexpr uint32_t kCellBlock = 128;
constexpr uint32_t kIntakeBlock = 256;
constexpr uint32_t kIntakePerThread = 4;

template <class J>
__device__ __forceinline__ uint32_t block_job(const J* __restrict__ jobs, uint32_t n_jobs) {
    __shared__ uint32_t s_j;
    if (threadIdx.x == 0) {
        uint32_t lo = 0, hi = n_jobs;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (jobs[mid].block0 <= blockIdx.x) lo = mid;
            else hi = mid;
        }
        s_j = lo;
    }
    __syncthreads();
    return s_j;
}

template <int ST>
__global__ void __launch_bounds__(kCellBlock)
    k_batch_cells(const CellJob* __restrict__ jobs, uint32_t n_jobs) {
    pdl_begin();
    const CellJob& J = jobs[block_job(jobs, n_jobs)];
    const uint32_t i = (blockIdx.x - J.block0) * kCellBlock + threadIdx.x;
    // Warp-cooperative steps keep every lane (a block's warps belong to one job).
    if (ST == ST_INHIB_MTP) {
        inhib_mtp_warp(J.axns, J.slices, J.L, J.radius, rnd_at(J.key, J.ctl->cycle),
                       rnd_at(J.L.rnd_key_ssc_mtp, J.ctl->cycle), J.learn != 0, i, i < J.n);
        return;
    }
    if (ST == ST_PYR_TAIL) {
        pyr_tail_warp(J.axns, J.slices, J.L, J.ctrl, J.learn != 0, J.ctl, i, i < J.n, J.tufts);
        return;
    }
    if (i >= J.n) return;
    switch (ST) {
    case ST_SSC_CYCLE: ssc_cycle_item(J.L, i); break;
    case ST_INHIB_SIMPLE: inhib_simple_item(J.axns, J.slices, J.L, J.radius, rnd_at(J.key, J.ctl->cycle), i); break;
    case ST_INHIB_PASS: inhib_passthrough_item(J.axns, J.slices, J.L, i); break;
    case ST_PYR_OUTPUT: pyr_output_item(J.axns, J.slices, J.L, i); break;
    case ST_INTRA_COL: intra_column_item(J.axns, J.slices, J.L, i); break;
    case ST_PYR_CYCLE: pyr_cycle_item(J.L, i); break;
    case ST_DST_MTP: tft_dst_mtp_item(J.axns, J.L, J.x, rnd_at(J.L.tft[J.x].rnd_key_mtp, J.ctl->cycle), i); break;
    case ST_SSC_MTP: ssc_mtp_item(J.axns, J.L, rnd_at(J.L.rnd_key_ssc_mtp, J.ctl->cycle), i); break;
    case BK_TUFT_CELLS:
        tuft_cell_item(J.axns, J.slices, J.L, J.x, rnd_at(J.L.tft[J.x].rnd_key_den, J.ctl->cycle), i);
        break;
    default: break;
    }
}

__global__ void __launch_bounds__(kIntakeBlock)
    k_batch_intake(const IntakeJob* __restrict__ jobs, uint32_t n_jobs, const BatchCtl* __restrict__ bc) {
    pdl_begin();
    const IntakeJob& J = jobs[block_job(jobs, n_jobs)];
    const uint8_t* src = J.src;
    if (!src) {
        if (!bc->frames) return;   // inputs as last written per area
        src = bc->frames + bc->cursor * bc->frame_bytes + J.src_off;
    }
    const uint32_t i0 = ((blockIdx.x - J.block0) * kIntakeBlock + threadIdx.x) * kIntakePerThread;
#pragma unroll
    for (uint32_t k = 0; k < kIntakePerThread; k++)
        if (i0 + k < J.len) J.dst[i0 + k] = src[i0 + k];
}

__global__ void k_batch_cycle_end(AreaCtl* const* __restrict__ ctls, uint32_t n, BatchCtl* bc) {
    pdl_begin();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) end_cycle(ctls[i]);
    if (i == 0) bc->cursor += 1;
}

__global__ void k_batch_begin(BatchCtl* bc, const uint8_t* frames, uint64_t frame_bytes) {
    bc->frames = frames;
    bc->cursor = 0;
    bc->frame_bytes = frame_bytes;
}

// Per-cell step kind -> launch.
// Every area's pyramidal tail: its own kernel at eight blocks of 128 per SM
// (64 registers, none spilled; 72 and seven blocks as an instantiation of
// k_batch_cells): a batch's tail covers every area's cells in several waves,
// and the extra block per SM took batch_64's tail from 0.120 to 0.084 ms.
__global__ void __launch_bounds__(kCellBlock, 8) k_batch_tail(const CellJob* __restrict__ jobs, uint32_t n_jobs) {
    pdl_begin();
    const CellJob& J = jobs[block_job(jobs, n_jobs)];
    const uint32_t i = (blockIdx.x - J.block0) * kCellBlock + threadIdx.x;
    pyr_tail_warp(J.axns, J.slices, J.L, J.ctrl, J.learn != 0, J.ctl, i, i < J.n, J.tufts);
}

void launch_cells(int st, const CellJob* jobs, uint32_t n_jobs, uint32_t n_blocks, cudaStream_t s) {
    if (!n_blocks) return;
    switch (st) {
#define BM_CELLS(K) \
    case K: launch_pdl(k_batch_cells<K>, n_blocks, kCellBlock, 0, s, jobs, n_jobs); break;
        BM_CELLS(ST_SSC_CYCLE)
        BM_CELLS(ST_INHIB_SIMPLE)
        BM_CELLS(ST_INHIB_PASS)
        BM_CELLS(ST_PYR_OUTPUT)
        BM_CELLS(ST_INTRA_COL)
        BM_CELLS(ST_PYR_CYCLE)
        BM_CELLS(ST_DST_MTP)
        BM_CELLS(ST_SSC_MTP)
        BM_CELLS(ST_INHIB_MTP)
    case ST_PYR_TAIL: launch_pdl(k_batch_tail, n_blocks, kCellBlock, 0, s, jobs, n_jobs); break;
        BM_CELLS(BK_TUFT_CELLS)
#undef BM_CELLS
    default: break;
    }
}

bool is_cell_step(int st) {
    return st == ST_SSC_CYCLE || st == ST_INHIB_SIMPLE || st == ST_INHIB_PASS || st == ST_PYR_OUTPUT ||
           st == ST_INTRA_COL || st == ST_PYR_CYCLE || st == ST_DST_MTP || st == ST_SSC_MTP ||
           st == ST_INHIB_MTP || st == ST_PYR_TAIL;
}

}  // namespace

struct bm_batch_s {
    enum Form { F_CELLS, F_FUSED, F_EACH, F_END, F_REGROW };
    struct CellLaunch {
        int kind;
        CellJob* d_jobs;
        uint32_t n_jobs, n_blocks;
    };
    // One step of the batch's schedule: the areas whose programs have it.
    struct StepPlan {
        Step st;
        std::vector<bm_area> areas;
        std::vector<std::pair<bm_area, uint32_t>> tufts;   // tuft steps: the (area, tuft) jobs
        Form form = F_EACH;
        std::vector<CellLaunch> cells;   // F_CELLS: launches in order
        FusedBatch fb;
        BatchShape shape;                // F_FUSED: ring stages and CTAs per SM (autotuned)
        bool side = false;               // runs on the side stream (no conflict with any earlier main step)
        std::vector<size_t> waits;       // side steps this main step must wait for
        RegrowJob* d_regrow = nullptr;   // F_REGROW: every area's regrowth jobs, one launch
        uint32_t n_regrow = 0, regrow_blocks = 0;
        // Profiling (eager cycles only): launches and device milliseconds.
        uint64_t prof_n = 0;
        double prof_ms = 0;
    };
    bm_ctx ctx = nullptr;
    std::vector<bm_area> areas;          // every area, in batch order
    std::vector<StepPlan> plan;          // the schedule: a common supersequence of the areas' programs
    uint32_t plan_launches = 0;
    bool profiling = false;
    struct Rec { size_t step; cudaEvent_t a, b; };
    std::vector<Rec> pending;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t ev() {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void drain_profile() {
        for (auto& r : pending) {
            float ms = 0.f;
            cudaEventSynchronize(r.b);
            cudaEventElapsedTime(&ms, r.a, r.b);
            plan[r.step].prof_n++;
            plan[r.step].prof_ms += ms;
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        pending.clear();
    }
    struct Tract {
        uint32_t src_area, src_output, dst_area, dst_input;
        uint64_t dst_off;
    };
    std::vector<Tract> tracts;
    IntakeJob* d_intake = nullptr;
    uint32_t n_intake = 0, intake_blocks = 0;
    uint64_t frame_bytes = 0;            // external inputs of one cycle
    BatchCtl* d_bctl = nullptr;
    AreaCtl** d_ctls = nullptr;
    bool use_graph = true;
    cudaStream_t cap = nullptr;          // private stream for graph capture
    // Side stream: tuft steps that depend on nothing earlier in the cycle
    // (e.g. the pyramidal distal tufts, which read only the previous cycle's
    // axons) run beside the main stream's chain of dependent steps.
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr;
    std::vector<cudaEvent_t> side_ev;    // per plan step (side steps only)
    size_t last_side = SIZE_MAX;
    bool detached = false;               // an area was destroyed first: the batch only waits to be freed
    std::vector<uint32_t> versions;      // each area's access_version when the schedule was made
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    cudaStream_t stream() const { return ctx->stream(); }
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
};

// The links between areas and the batches holding them (bm_area_s::batches
// and n_batches). A batch may be destroyed on another thread than the one
// creating the next batch over the same areas (a server's builder thread).
static std::mutex g_links;

// An area being destroyed leaves every batch holding it: the batch keeps
// nothing that points into the area and will not cycle again.
void bm::detach_from_batches(bm_area_s* A) {
    std::lock_guard<std::mutex> lk(g_links);
    for (bm_batch_s* B : A->batches) {
        DevGuard g(B->ctx->device);
        cudaStreamSynchronize(B->stream());
        B->drop_graph();
        for (bm_area& X : B->areas)
            if (X == A) X = nullptr;
        B->detached = true;
    }
    A->batches.clear();
    A->n_batches = 0;
}

namespace {

void free_plan(bm_batch_s* B) {
    const bool pl = B->ctx->pool != nullptr;
    for (auto& p : B->plan) {
        for (auto& c : p.cells) dev_free(c.d_jobs, pl, B->stream());
        dev_free(p.d_regrow, pl, B->stream());
        free_fused_batch(p.fb);
    }
    B->plan.clear();
}

void free_batch(bm_batch_s* B) {
    if (!B) return;
    DevGuard g(B->ctx->device);
    // Areas destroyed before the batch were detached (their entries are null).
    {
        std::lock_guard<std::mutex> lk(g_links);
        for (bm_area A : B->areas) {
            if (!A) continue;
            if (A->n_batches) A->n_batches--;
            A->batches.erase(std::remove(A->batches.begin(), A->batches.end(), B), A->batches.end());
        }
    }
    B->drop_graph();
    free_plan(B);
    const bool pl = B->ctx->pool != nullptr;
    dev_free(B->d_intake, pl, B->stream());
    dev_free(B->d_bctl, pl, B->stream());
    dev_free(B->d_ctls, pl, B->stream());
    if (B->cap) cudaStreamDestroy(B->cap);
    if (B->side) cudaStreamDestroy(B->side);
    if (B->ev_fork) cudaEventDestroy(B->ev_fork);
    for (cudaEvent_t e : B->side_ev)
        if (e) cudaEventDestroy(e);
    for (auto& r : B->pending) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (auto e : B->pool) cudaEventDestroy(e);
    ctx_release(B->ctx);
    delete B;
}

// Work items of a per-cell launch of kind k for step st of area A.
uint64_t items_of(const bm_area_s* A, int k, const Step& st) {
    const bm_layer_plan& L = A->plan.layers[st.layer];
    switch (k) {
    case ST_INTRA_COL: return (uint64_t)L.v_size * L.u_size;
    case ST_PYR_TAIL: return tail_items(L.depth, L.v_size * L.u_size);
    default: return L.cells;
    }
}

// One batched per-cell launch of kind k for step st over every area.
int add_cells(bm_ctx ctx, bm_batch_s::StepPlan& p, int k) {
    const Step& st = p.st;
    std::vector<CellJob> jobs;
    uint64_t blocks = 0;
    for (bm_area A : p.areas) {
        CellJob J;
        std::memset(&J, 0, sizeof J);
        J.L = A->dl[st.layer];
        J.axns = A->axns();
        J.slices = A->slices;
        J.ctl = A->ctl;
        J.x = st.idx;
        if (k == ST_INHIB_SIMPLE || k == ST_INHIB_MTP) {
            J.key = A->inhib_key[st.layer][st.idx];
            J.radius = (int32_t)A->plan.layers[st.layer].ctrl[st.idx].field_radius;
        }
        if (k == ST_PYR_TAIL) {
            J.ctrl = st.idx == 0xFF ? 0 : (A->plan.layers[st.layer].ctrl[st.idx].kind == BM_LYR_CTRL_INTRA_COLUMN ? 1 : 2);
            J.tufts = st.tufts;
        }
        J.learn = st.arg;
        const uint64_t n = items_of(A, k, st);
        if (n > 0xFFFFFFFFull) return set_err(BM_ERR_UNSUPPORTED, "batched step of more than 2^32 items");
        J.n = (uint32_t)n;
        J.block0 = (uint32_t)blocks;
        blocks += (n + kCellBlock - 1) / kCellBlock;
        jobs.push_back(J);
    }
    if (blocks > 0x7FFFFFFFull) return set_err(BM_ERR_UNSUPPORTED, "batched step of too many blocks");
    bm_batch_s::CellLaunch c{k, nullptr, (uint32_t)jobs.size(), (uint32_t)blocks};
    cudaError_t e = dev_alloc(ctx, &c.d_jobs, jobs.size() * sizeof(CellJob));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c.d_jobs, jobs.data(), jobs.size() * sizeof(CellJob), cudaMemcpyHostToDevice, ctx->stream());
    if (e != cudaSuccess) {
        dev_free(c.d_jobs, ctx->pool != nullptr, ctx->stream());
        return cuda_err(e, "batched step jobs");
    }
    p.cells.push_back(c);
    p.form = bm_batch_s::F_CELLS;
    return BM_OK;
}

int build_fused(bm_batch_s::StepPlan& p) {
    std::vector<FusedJob> jobs;
    for (auto& [A, t] : p.tufts) {
        if (!A->fused.t[p.st.layer][t].ok) return BM_OK;
        jobs.push_back({&A->fused, &A->dl[p.st.layer], A->axns(), A->slices, A->ctl, p.st.layer, t,
                        (p.st.arg & 1) != 0});
    }
    int rc = prepare_fused_batch(p.fb, jobs, p.shape);
    if (rc != BM_OK) return rc;
    p.form = p.fb.ok ? bm_batch_s::F_FUSED : bm_batch_s::F_EACH;
    return BM_OK;
}

// Every area's regrowth jobs in one table (block0 rebased), one launch.
int build_regrow(bm_ctx ctx, bm_batch_s::StepPlan& p) {
    std::vector<RegrowJob> jobs;
    uint64_t blocks = 0;
    for (bm_area A : p.areas)
        for (RegrowJob J : A->regrow) {
            J.block0 = (uint32_t)blocks;
            blocks += (J.n + kRegrowBlock - 1) / kRegrowBlock;
            jobs.push_back(J);
        }
    if (blocks > 0x7FFFFFFFull) return set_err(BM_ERR_UNSUPPORTED, "batched regrowth of too many blocks");
    if (jobs.empty()) {
        p.form = bm_batch_s::F_END;
        return BM_OK;
    }
    cudaError_t e = dev_alloc(ctx, &p.d_regrow, jobs.size() * sizeof(RegrowJob));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p.d_regrow, jobs.data(), jobs.size() * sizeof(RegrowJob), cudaMemcpyHostToDevice,
                            ctx->stream());
    if (e != cudaSuccess) return cuda_err(e, "batched regrowth jobs");
    p.n_regrow = (uint32_t)jobs.size();
    p.regrow_blocks = (uint32_t)blocks;
    p.form = bm_batch_s::F_REGROW;
    return BM_OK;
}

int build_step(bm_ctx ctx, bm_batch_s::StepPlan& p) {
    const Step& st = p.st;
    if (st.kind == ST_CYCLE_END) {
        p.form = bm_batch_s::F_END;
        return BM_OK;
    }
    if (st.kind == ST_REGROW) return build_regrow(ctx, p);
    if (is_cell_step(st.kind)) return add_cells(ctx, p, st.kind);
    if (st.kind != ST_TUFT) return BM_OK;   // the plain form's whole-layer tuft stages: each area's own
    p.tufts.clear();
    for (bm_area A : p.areas) p.tufts.push_back({A, st.idx});
    bool none_ok = true, all_ok = true;
    for (auto& [A, t] : p.tufts) {
        const bool ok = A->fused.t[st.layer][t].ok;
        none_ok = none_ok && !ok;
        all_ok = all_ok && ok;
    }
    if (all_ok) {
        // Tile size from the whole step's work, not each area's own: one
        // launch serves every area, so small areas need not cut tiny tiles
        // to fill the device (the autotuner refines this).
        uint64_t total = 0;
        int sms = 148;
        for (auto& [A, t] : p.tufts) {
            const bm_layer_plan& L = A->plan.layers[st.layer];
            total += (uint64_t)L.cells * L.tufts[t].syns_per_tft;
            sms = A->fused.sms;
        }
        // A power of two, so that batches rebuilt as areas come and go keep
        // their tiles (and compiled offsets) until the work doubles or halves.
        uint64_t want = std::min<uint64_t>(65536, std::max<uint64_t>(4096, total / ((uint64_t)sms * 16)));
        uint32_t target = 4096;
        while ((uint64_t)target * 2 <= want) target *= 2;
        for (auto& [A, t] : p.tufts) {
            FusedTuft& FT = A->fused.t[st.layer][t];
            // An autotuned choice stays; an area another batch also holds
            // keeps its tiles (that batch's launches are planned on them).
            if (!FT.tiled || FT.tile_tuned || FT.tile_target == target || A->n_batches > 1) continue;
            bool changed = false;
            if (retile_fused_tuft(A->fused, A->plan, st.layer, t, target, &changed, FT.fp_staged) && changed)
                A->verify_pending[st.layer] = true;
        }
        return build_fused(p);
    }
    if (!none_ok) return BM_OK;
    // No area can take the fused kernel here (e.g. one-synapse dendrites):
    // the tuft's four stages per cell, batched.
    return add_cells(ctx, p, BK_TUFT_CELLS);
}

// Consecutive batched tuft steps of one layer touch disjoint buffers: one
// launch serves all their (area, tuft) jobs.
int merge_tuft_steps(bm_batch_s* B) {
    std::vector<bm_batch_s::StepPlan> out;
    for (auto& p : B->plan) {
        if (!out.empty() && p.form == bm_batch_s::F_FUSED && out.back().form == bm_batch_s::F_FUSED &&
            p.st.kind == ST_TUFT && out.back().st.kind == ST_TUFT && p.st.layer == out.back().st.layer &&
            p.st.arg == out.back().st.arg) {
            auto& q = out.back();
            q.tufts.insert(q.tufts.end(), p.tufts.begin(), p.tufts.end());
            for (bm_area A : p.areas)
                if (std::find(q.areas.begin(), q.areas.end(), A) == q.areas.end()) q.areas.push_back(A);
            free_fused_batch(p.fb);
            int rc = build_fused(q);
            if (rc != BM_OK) return rc;
            continue;
        }
        out.push_back(p);
    }
    B->plan.swap(out);
    return BM_OK;
}

void count_launches(bm_batch_s* B) {
    uint32_t n = 0;
    for (const auto& p : B->plan) {
        const Step& st = p.st;
        if (p.form == bm_batch_s::F_EACH) {
            // Each area's own launches for this step.
            for (bm_area A : p.areas) {
                const bm_layer_plan& L = A->plan.layers[st.layer];
                uint32_t per = 1;
                if (st.kind == ST_TUFTS_PLAIN) per = 1 + 2 * L.n_tufts + (L.kind == BM_LYR_PYRAMIDAL ? L.n_tufts : 0);
                if (st.kind == ST_SMOOTH) per = 6;
                if (st.kind == ST_FILTER) per = A->plan.filter_chains[st.idx].n_filters;
                n += per;
            }
        } else if (p.form == bm_batch_s::F_CELLS) {
            n += (uint32_t)p.cells.size();
        } else if (p.form == bm_batch_s::F_FUSED) {
            n += (uint32_t)p.fb.params.size();
        } else if (p.form == bm_batch_s::F_REGROW) {
            n += 1;
        }
    }
    B->plan_launches = n;
}

// The accesses of plan step p for area A (a merged tuft step: every tuft of
// A in it).
StepAccess plan_access(const bm_batch_s::StepPlan& p, bm_area A) {
    if (p.st.kind == ST_TUFT && !p.tufts.empty()) {
        StepAccess a;
        for (auto& [B, t] : p.tufts)
            if (B == A) a |= step_access(A, p.st, (int)t);
        return a;
    }
    return step_access(A, p.st);
}

// Splits the schedule over two streams: a tuft step whose accesses conflict,
// in no area, with any earlier step left on the main stream goes to the side
// stream (side steps keep their order there); a main step waits for every
// earlier side step it conflicts with, and the cycle end for all of them.
int schedule_side(bm_batch_s* B) {
    const size_t n = B->plan.size();
    B->last_side = SIZE_MAX;
    B->versions.clear();
    for (bm_area A : B->areas) B->versions.push_back(A->access_version);
    std::vector<std::vector<std::pair<bm_area, StepAccess>>> acc(n);
    for (size_t k = 0; k < n; k++)
        for (bm_area A : B->plan[k].areas) acc[k].push_back({A, plan_access(B->plan[k], A)});
    auto clash = [&](size_t j, size_t k) {
        for (auto& [a, x] : acc[j])
            for (auto& [b, y] : acc[k])
                if (a == b && conflict(x, y)) return true;
        return false;
    };
    for (size_t k = 0; k < n; k++) {
        auto& p = B->plan[k];
        p.side = false;
        p.waits.clear();
        if ((p.st.kind != ST_TUFT && p.st.kind != ST_TUFTS_PLAIN) || p.form == bm_batch_s::F_END) continue;
        bool free = true;
        for (size_t j = 0; j < k && free; j++)
            if (!B->plan[j].side && clash(j, k)) free = false;
        p.side = free;
    }
    for (size_t k = 0; k < n; k++) {
        if (B->plan[k].side) {
            B->last_side = k;
            continue;
        }
        for (size_t j = 0; j < k; j++)
            if (B->plan[j].side && clash(j, k)) B->plan[k].waits.push_back(j);
    }
    if (B->last_side == SIZE_MAX) return BM_OK;
    cudaError_t e = cudaSuccess;
    if (!B->side) e = stream_like(B->stream(), &B->side);
    if (e == cudaSuccess && !B->ev_fork) e = cudaEventCreateWithFlags(&B->ev_fork, cudaEventDisableTiming);
    for (cudaEvent_t ev : B->side_ev)
        if (ev) cudaEventDestroy(ev);
    B->side_ev.assign(n, nullptr);
    for (size_t k = 0; k < n && e == cudaSuccess; k++)
        if (B->plan[k].side) e = cudaEventCreateWithFlags(&B->side_ev[k], cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_err(e, "side stream");
    return BM_OK;
}

// The schedule: the shortest common supersequence of the areas' stage
// programs (merged one distinct program at a time through their longest
// common subsequence), each step run over the areas that have it. Areas are
// independent, so any order that keeps each area's own order is exact. The
// cycle-end step is done once for the whole batch.
int build_plan(bm_batch_s* B) {
    free_plan(B);
    // Each area's program, with per-cell tufts folded into the tails only
    // while the batch's cells with such tufts stay within kFoldCellTufts.
    uint64_t cells = 0;
    for (bm_area A : B->areas) cells += cell_tuft_cells(A);
    std::vector<std::vector<Step>> progs(B->areas.size());
    for (size_t a = 0; a < B->areas.size(); a++) area_steps(B->areas[a], progs[a], cells <= kFoldCellTufts);
    std::vector<Step> U;
    std::vector<std::vector<uint32_t>> who;   // who[k]: areas (batch indices) having U[k]
    for (uint32_t a = 0; a < B->areas.size(); a++) {
        const std::vector<Step>& P = progs[a];
        // Same program as an earlier area: its positions in U are known.
        bool placed = false;
        for (uint32_t b = 0; b < a && !placed; b++) {
            if (!(progs[b] == P)) continue;
            for (auto& w : who)
                if (std::find(w.begin(), w.end(), b) != w.end()) w.push_back(a);
            placed = true;
        }
        if (placed) continue;
        const size_t n = U.size(), m = P.size();
        std::vector<std::vector<uint16_t>> L(n + 1, std::vector<uint16_t>(m + 1, 0));
        for (size_t i = n; i-- > 0;)
            for (size_t j = m; j-- > 0;)
                L[i][j] = (U[i] == P[j]) ? (uint16_t)(L[i + 1][j + 1] + 1) : std::max(L[i + 1][j], L[i][j + 1]);
        std::vector<Step> U2;
        std::vector<std::vector<uint32_t>> who2;
        size_t i = 0, j = 0;
        while (i < n || j < m) {
            if (i < n && j < m && U[i] == P[j]) {
                U2.push_back(U[i]);
                who2.push_back(who[i]);
                who2.back().push_back(a);
                i++, j++;
            } else if (j == m || (i < n && L[i + 1][j] >= L[i][j + 1])) {
                U2.push_back(U[i]);
                who2.push_back(who[i]);
                i++;
            } else {
                U2.push_back(P[j]);
                who2.push_back({a});
                j++;
            }
        }
        U.swap(U2);
        who.swap(who2);
    }
    for (size_t k = 0; k < U.size(); k++) {
        bm_batch_s::StepPlan p;
        p.st = U[k];
        for (uint32_t a : who[k]) p.areas.push_back(B->areas[a]);
        int rc = p.st.kind == ST_CYCLE_END ? (p.form = bm_batch_s::F_END, BM_OK) : build_step(B->ctx, p);
        B->plan.push_back(p);
        if (rc != BM_OK) return rc;
    }
    int rc = merge_tuft_steps(B);
    if (rc != BM_OK) return rc;
    count_launches(B);
    return schedule_side(B);
}

// The head-of-cycle copies: every tract, then every input of every area that
// no tract feeds, taken from the frame block in (area, input) order.
int build_intake(bm_batch_s* B) {
    dev_free(B->d_intake, B->ctx->pool != nullptr, B->stream());
    B->d_intake = nullptr;
    B->n_intake = B->intake_blocks = 0;
    B->frame_bytes = 0;
    std::vector<IntakeJob> jobs;
    uint64_t blocks = 0;
    const uint32_t per_block = kIntakeBlock * kIntakePerThread;
    auto add = [&](IntakeJob J) {
        J.block0 = (uint32_t)blocks;
        blocks += (J.len + per_block - 1) / per_block;
        jobs.push_back(J);
    };
    // A filtered source's bytes land in its chain's first buffer.
    std::vector<FramePiece> pieces;
    for (const auto& T : B->tracts) {
        bm_area S = B->areas[T.src_area], D = B->areas[T.dst_area];
        frame_pieces(D, T.dst_input, T.dst_off, S->plan.outputs[T.src_output].len, pieces);
        for (const FramePiece& p : pieces) {
            IntakeJob J{};
            J.dst = p.dst;
            J.src = S->axns() + S->plan.outputs[T.src_output].axn_idz + p.off;
            J.len = p.len;
            add(J);
        }
    }
    for (uint32_t a = 0; a < B->areas.size(); a++) {
        bm_area A = B->areas[a];
        for (uint32_t i = 0; i < A->plan.n_inputs; i++) {
            bool fed = false;
            for (const auto& T : B->tracts) fed = fed || (T.dst_area == a && T.dst_input == i);
            if (fed) continue;
            frame_pieces(A, i, 0, A->plan.inputs[i].len, pieces);
            for (const FramePiece& p : pieces) {
                IntakeJob J{};
                J.dst = p.dst;
                J.src_off = B->frame_bytes + p.off;
                J.len = p.len;
                add(J);
            }
            B->frame_bytes += A->plan.inputs[i].len;
        }
    }
    if (jobs.empty()) return BM_OK;
    if (blocks > 0x7FFFFFFFull) return set_err(BM_ERR_UNSUPPORTED, "batched intake too large");
    cudaError_t e = dev_alloc(B->ctx, &B->d_intake, jobs.size() * sizeof(IntakeJob));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(B->d_intake, jobs.data(), jobs.size() * sizeof(IntakeJob), cudaMemcpyHostToDevice,
                            B->stream());
    if (e != cudaSuccess) return cuda_err(e, "batched intake jobs");
    B->n_intake = (uint32_t)jobs.size();
    B->intake_blocks = (uint32_t)blocks;
    return BM_OK;
}

void enqueue_batch_cycle(bm_batch_s* B, cudaStream_t main) {
    if (B->intake_blocks)
        launch_pdl(k_batch_intake, B->intake_blocks, kIntakeBlock, 0, main, B->d_intake, B->n_intake, B->d_bctl);
    const bool prof = B->profiling && main != B->cap;
    // Profiling times each step on its own: everything on the main stream.
    const bool fork = !prof && B->last_side != SIZE_MAX;
    if (fork) {
        cudaEventRecord(B->ev_fork, main);
        cudaStreamWaitEvent(B->side, B->ev_fork, 0);
    }
    for (size_t k = 0; k < B->plan.size(); k++) {
        auto& p = B->plan[k];
        const bool on_side = fork && p.side;
        cudaStream_t s = on_side ? B->side : main;
        if (fork && !on_side)
            for (size_t j : p.waits) cudaStreamWaitEvent(main, B->side_ev[j], 0);
        bm_batch_s::Rec r{k, nullptr, nullptr};
        if (prof && p.form != bm_batch_s::F_END) {
            r.a = B->ev();
            r.b = B->ev();
            cudaEventRecord(r.a, s);
        }
        switch (p.form) {
        case bm_batch_s::F_CELLS:
            for (auto& c : p.cells) launch_cells(c.kind, c.d_jobs, c.n_jobs, c.n_blocks, s);
            break;
        case bm_batch_s::F_FUSED: launch_fused_batch(p.fb, s); break;
        case bm_batch_s::F_REGROW: launch_regrow(p.d_regrow, p.n_regrow, p.regrow_blocks, s); break;
        case bm_batch_s::F_END: break;
        default:
            for (bm_area A : p.areas) exec_step(A, p.st, s);
            break;
        }
        if (r.a) {
            cudaEventRecord(r.b, s);
            B->pending.push_back(r);
        }
        if (on_side) cudaEventRecord(B->side_ev[k], B->side);
    }
    if (fork) cudaStreamWaitEvent(main, B->side_ev[B->last_side], 0);   // the side stream rejoins
    const uint32_t n = (uint32_t)B->areas.size();
    launch_pdl(k_batch_cycle_end, (n + 127) / 128, 128, 0, main, B->d_ctls, n, B->d_bctl);
}

int ensure_graph(bm_batch_s* B) {
    if (B->exec) return BM_OK;
    cudaError_t e = cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_err(e, "cudaStreamBeginCapture");
    enqueue_batch_cycle(B, B->cap);
    e = cudaStreamEndCapture(B->cap, &B->graph);
    if (e != cudaSuccess) {
        B->graph = nullptr;
        return cuda_err(e, "cudaStreamEndCapture");
    }
    e = cudaGraphInstantiate(&B->exec, B->graph, 0);
    if (e != cudaSuccess) {
        B->drop_graph();
        return cuda_err(e, "cudaGraphInstantiate");
    }
    return BM_OK;
}

// After each batched cycle: every area's cycle count, then its samplers.
int after_cycle(bm_batch_s* B, cudaStream_t s) {
    for (bm_area A : B->areas) {
        A->host_cycle++;
        if (!A->samplers.empty()) {
            const int rc = sample_after_cycle(A, s);
            if (rc != BM_OK) return rc;
        }
    }
    return BM_OK;
}

int run_cycles(bm_batch_s* B, const void* frames, uint32_t n_cycles, bool refuse_after_errors = true) {
    if (B->detached) return set_err(BM_ERR_INVALID, "an area of this batch was destroyed");
    // An area whose earlier cycle ended with device error bits stops the batch
    // (bm_area_clear_errors on that area re-enables it).
    for (size_t a = 0; a < B->areas.size() && refuse_after_errors; a++)
        if (const unsigned int e = B->areas[a]->seen_errors())
            return set_err(BM_ERR_TIMEOUT, "area %zu of the batch ended an earlier cycle with device error bits 0x%x",
                           a, e);
    cudaStream_t s = B->stream();
    for (bm_area A : B->areas) run_pending_verifies(A, s);
    // Caller writes may have changed what an area's tuft steps read.
    for (size_t a = 0; a < B->areas.size(); a++)
        if (a >= B->versions.size() || B->areas[a]->access_version != B->versions[a]) {
            B->drop_graph();
            const int rc = schedule_side(B);
            if (rc != BM_OK) return rc;
            break;
        }
    k_batch_begin<<<1, 1, 0, s>>>(B->d_bctl, (const uint8_t*)frames, B->frame_bytes);
    if (B->use_graph && !B->profiling) {
        int rc = ensure_graph(B);
        if (rc != BM_OK) return rc;
        for (uint32_t k = 0; k < n_cycles; k++) {
            cudaError_t e = cudaGraphLaunch(B->exec, s);
            if (e != cudaSuccess) return cuda_err(e, "cudaGraphLaunch");
            const int rc = after_cycle(B, s);
            if (rc != BM_OK) return rc;
        }
    } else {
        for (uint32_t k = 0; k < n_cycles; k++) {
            enqueue_batch_cycle(B, s);
            const int rc = after_cycle(B, s);
            if (rc != BM_OK) return rc;
        }
    }
    // An area cycling on its own later starts its front stream after these.
    for (bm_area A : B->areas) A->mark_main();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_err(e, "batched cycle");
    return BM_OK;
}

// --------------------------------------------------------- autotuner -----
// The buffers one tuft step writes, per area: synapse states and flags,
// dendrite raw states, states and activities, (pyramidal) the eight
// cell-tuft buffers, and (spiny stellate, ssc_cycle folded in) the cell
// energies.
struct Range {
    uint8_t* p;
    uint64_t n;
};
void step_ranges(bm_area_s* A, uint32_t i, uint32_t t, bool ssc_soma, std::vector<Range>& out) {
    const bm_layer_plan& L = A->plan.layers[i];
    const bm_tuft_plan& T = L.tufts[t];
    auto add = [&](int k, uint64_t off, uint64_t n) { out.push_back({A->slab + L.buf_off[k] + off, n}); };
    const uint64_t ns = (uint64_t)L.cells * T.syns_per_tft, nd = (uint64_t)L.cells * T.dens_per_tft;
    add(BM_BUF_SYN_STATES, T.syn_idz, ns);
    add(BM_BUF_SYN_FLAG_SETS, T.syn_idz, ns);
    add(BM_BUF_DEN_STATES_RAW, T.den_idz, nd);
    add(BM_BUF_DEN_STATES, T.den_idz, nd);
    add(BM_BUF_DEN_ACTIVITIES, T.den_idz, nd);
    if (L.kind == BM_LYR_PYRAMIDAL)
        for (int k = BM_BUF_TFT_PREV_BEST_DEN_IDS; k <= BM_BUF_TFT_STATES; k++) add(k, T.cel_idz, L.cells);
    if (ssc_soma && L.kind == BM_LYR_SPINY_STELLATE && L.buf_off[BM_BUF_CEL_ENERGIES] != UINT64_MAX)
        add(BM_BUF_CEL_ENERGIES, 0, L.cells);
}

std::string step_key(const bm_batch_s::StepPlan& p) {
    std::string k = "L" + std::to_string(p.st.layer);
    for (auto& [A, t] : p.tufts) {
        const bm_layer_plan& L = A->plan.layers[p.st.layer];
        const bm_tuft_plan& T = L.tufts[t];
        char buf[96];
        snprintf(buf, sizeof buf, ":T%u:%ux%ux%u/%u/%u/%u", t, L.v_size, L.u_size, L.depth, T.syns_per_tft,
                 T.syns_per_den, T.n_src_uniq);
        k += buf;
    }
    return k;
}

// A step's tuned launch: synapses per tile, its BatchShape, and whether the
// consumers stage the footprints (1) rather than load them as tensor boxes.
struct Tuned {
    uint32_t target = 0, stages = 0, ctas = 0, staged = 0;
};

// One line per step: its key, the tile target, the ring's most stages, the
// CTAs per SM and the footprint form (fields left out read as 0).
std::map<std::string, Tuned> read_cache(const char* path) {
    std::map<std::string, Tuned> m;
    if (!path) return m;
    FILE* f = fopen(path, "r");
    if (!f) return m;
    char line[4300], key[4096];
    while (fgets(line, sizeof line, f)) {
        Tuned v;
        if (sscanf(line, "%4095s %u %u %u %u", key, &v.target, &v.stages, &v.ctas, &v.staged) >= 2 && v.target)
            m[key] = v;
    }
    fclose(f);
    return m;
}

void write_cache(const char* path, const std::map<std::string, Tuned>& m) {
    if (!path) return;
    FILE* f = fopen(path, "w");
    if (!f) return;
    for (auto& kv : m)
        fprintf(f, "%s %u %u %u %u\n", kv.first.c_str(), kv.second.target, kv.second.stages, kv.second.ctas,
                kv.second.staged);
    fclose(f);
}

// Retiles tuft (i, t) of every area for `target` synapses per tile (with
// footprints staged by the consumers when `staged`) and rebuilds the step's
// batched launch. False when some area cannot take it.
bool apply_target(bm_batch_s* B, bm_batch_s::StepPlan& p, uint32_t target, bool staged = false) {
    for (auto& [A, t] : p.tufts)
        if (A->n_batches > 1) return false;   // another batch's launches are planned on these tiles
    for (auto& [A, t] : p.tufts) {
        bool changed = false;
        if (!retile_fused_tuft(A->fused, A->plan, p.st.layer, t, target, &changed, staged)) return false;
        A->fused.t[p.st.layer][t].tile_tuned = true;
        if (changed) A->verify_pending[p.st.layer] = true;
    }
    for (bm_area A : p.areas) run_pending_verifies(A, B->stream());
    return build_fused(p) == BM_OK && p.form == bm_batch_s::F_FUSED;
}

}  // namespace

int bm::batch_cycle_frames_unchecked(bm_batch_s* B, const void* dev_frames) {
    DevGuard g(B->ctx->device);
    return run_cycles(B, dev_frames, 1, false);
}

extern "C" {

int bm_batch_create(bm_ctx ctx, const bm_area* areas, uint32_t n_areas, bm_batch* out) {
    if (!ctx || !areas || !out || n_areas == 0) return set_err(BM_ERR_INVALID, "bm_batch_create: null argument or no areas");
    *out = nullptr;
    for (uint32_t a = 0; a < n_areas; a++) {
        if (!areas[a]) return set_err(BM_ERR_INVALID, "bm_batch_create: area %u is null", a);
        if (areas[a]->ctx != ctx) return set_err(BM_ERR_INVALID, "bm_batch_create: area %u belongs to another context", a);
        for (uint32_t b = 0; b < a; b++)
            if (areas[b] == areas[a]) return set_err(BM_ERR_INVALID, "bm_batch_create: area %u appears twice", a);
    }
    DevGuard g(ctx->device);
    bm_batch_s* B = new (std::nothrow) bm_batch_s;
    if (!B) return set_err(BM_ERR_OOM, "host allocation failed");
    B->ctx = ctx;
    ctx_retain(ctx);
    B->areas.assign(areas, areas + n_areas);
    {
        std::lock_guard<std::mutex> lk(g_links);
        for (bm_area A : B->areas) {
            A->n_batches++;
            A->batches.push_back(B);
        }
    }
    cudaError_t e = stream_like(ctx->stream(), &B->cap);
    if (e != cudaSuccess) { free_batch(B); return cuda_err(e, "cudaStreamCreate"); }

    std::vector<AreaCtl*> ctls;
    for (bm_area A : B->areas) ctls.push_back(A->ctl);
    e = dev_alloc(ctx, &B->d_bctl, sizeof(BatchCtl));
    if (e == cudaSuccess) e = cudaMemsetAsync(B->d_bctl, 0, sizeof(BatchCtl), ctx->stream());
    if (e == cudaSuccess) e = dev_alloc(ctx, &B->d_ctls, ctls.size() * sizeof(AreaCtl*));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(B->d_ctls, ctls.data(), ctls.size() * sizeof(AreaCtl*), cudaMemcpyHostToDevice,
                            ctx->stream());
    if (e != cudaSuccess) { free_batch(B); return cuda_err(e, "batch set-up"); }
    int rc = build_intake(B);
    if (rc == BM_OK) rc = build_plan(B);
    // The job tables went up in order on the context's stream; a batch on a
    // pooled context (a server's) is cycled on that stream, any other may be
    // cycled on another stream once the caller changes it.
    if (rc == BM_OK && !ctx->pool) e = cudaStreamSynchronize(ctx->stream());
    if (rc == BM_OK && e != cudaSuccess) rc = cuda_err(e, "batch set-up");
    if (rc != BM_OK) { free_batch(B); return rc; }
    *out = B;
    return BM_OK;
}

int bm_batch_destroy(bm_batch batch) {
    if (!batch) return BM_OK;
    {
        DevGuard g(batch->ctx->device);
        cudaStreamSynchronize(batch->stream());
    }
    free_batch(batch);
    return BM_OK;
}

int bm_batch_set_graph(bm_batch batch, int on) {
    if (batch && batch->detached) return set_err(BM_ERR_INVALID, "an area of this batch was destroyed");
    if (!batch) return set_err(BM_ERR_INVALID, "null batch");
    batch->use_graph = on != 0;
    return BM_OK;
}

int bm_batch_cycle(bm_batch batch, uint32_t n_cycles) {
    if (!batch) return set_err(BM_ERR_INVALID, "null batch");
    DevGuard g(batch->ctx->device);
    return run_cycles(batch, nullptr, n_cycles);
}

int bm_batch_frame_bytes(bm_batch batch, uint64_t* out) {
    if (batch && batch->detached) return set_err(BM_ERR_INVALID, "an area of this batch was destroyed");
    if (!batch || !out) return set_err(BM_ERR_INVALID, "null argument");
    *out = batch->frame_bytes;
    return BM_OK;
}

int bm_batch_connect(bm_batch batch, uint32_t src_area, uint32_t src_output, uint32_t dst_area, uint32_t dst_input,
                     uint64_t dst_offset) {
    if (batch && batch->detached) return set_err(BM_ERR_INVALID, "an area of this batch was destroyed");
    if (!batch) return set_err(BM_ERR_INVALID, "null batch");
    bm_batch_s* B = batch;
    const uint32_t n = (uint32_t)B->areas.size();
    if (src_area >= n || dst_area >= n) return set_err(BM_ERR_INVALID, "bm_batch_connect: area index out of range");
    const bm_area_plan& S = B->areas[src_area]->plan;
    const bm_area_plan& D = B->areas[dst_area]->plan;
    if (src_output >= S.n_outputs) return set_err(BM_ERR_INVALID, "bm_batch_connect: output %u out of range", src_output);
    if (dst_input >= D.n_inputs) return set_err(BM_ERR_INVALID, "bm_batch_connect: input %u out of range", dst_input);
    const uint64_t len = S.outputs[src_output].len;
    if (dst_offset > D.inputs[dst_input].len || len > D.inputs[dst_input].len - dst_offset)
        return set_err(BM_ERR_INVALID,
                       "bm_batch_connect: %llu output axons at offset %llu overrun input %u of area %u (%u axons)",
                       (unsigned long long)len, (unsigned long long)dst_offset, dst_input, dst_area,
                       D.inputs[dst_input].len);
    for (const auto& T : B->tracts)
        if (T.dst_area == dst_area && T.dst_input == dst_input && dst_offset < T.dst_off + B->areas[T.src_area]->plan.outputs[T.src_output].len &&
            T.dst_off < dst_offset + len)
            return set_err(BM_ERR_INVALID, "bm_batch_connect: overlaps an existing tract into that input");
    DevGuard g(B->ctx->device);
    B->tracts.push_back({src_area, src_output, dst_area, dst_input, dst_offset});
    B->drop_graph();
    int rc = build_intake(B);
    if (rc != BM_OK) {
        B->tracts.pop_back();
        build_intake(B);
        return rc;
    }
    if (!B->ctx->pool) {
        const cudaError_t e = cudaStreamSynchronize(B->stream());
        if (e != cudaSuccess) return cuda_err(e, "tract intake tables");
    }
    return BM_OK;
}

int bm_batch_cycle_frames_device(bm_batch batch, const void* dev_frames, uint32_t n_cycles) {
    if (!batch || !dev_frames) return set_err(BM_ERR_INVALID, "null argument");
    if (!batch->frame_bytes) return set_err(BM_ERR_INVALID, "the batch has no input that a tract does not feed");
    DevGuard g(batch->ctx->device);
    return run_cycles(batch, dev_frames, n_cycles);
}

int bm_batch_set_profiling(bm_batch batch, int on) {
    if (batch && batch->detached) return set_err(BM_ERR_INVALID, "an area of this batch was destroyed");
    if (!batch) return set_err(BM_ERR_INVALID, "null batch");
    batch->profiling = on != 0;
    return BM_OK;
}

int bm_batch_get_profile(bm_batch batch, uint32_t n_max, uint32_t* kinds, uint32_t* layers, uint32_t* idx,
                         uint32_t* n_areas, uint64_t* launches, double* ms, uint32_t* n_out) {
    if (batch && batch->detached) return set_err(BM_ERR_INVALID, "an area of this batch was destroyed");
    if (!batch || !n_out) return set_err(BM_ERR_INVALID, "null argument");
    DevGuard g(batch->ctx->device);
    batch->drain_profile();
    uint32_t n = 0;
    for (auto& p : batch->plan) {
        if (!p.prof_n || n >= n_max) continue;
        if (kinds) kinds[n] = p.form == bm_batch_s::F_FUSED ? 1000u + p.st.kind : p.st.kind;
        if (layers) layers[n] = p.st.layer;
        if (idx) idx[n] = p.st.idx;
        if (n_areas) n_areas[n] = (uint32_t)p.areas.size();
        if (launches) launches[n] = p.prof_n;
        if (ms) ms[n] = p.prof_ms;
        n++;
    }
    *n_out = n;
    return BM_OK;
}

int bm_batch_reset_profile(bm_batch batch) {
    if (batch && batch->detached) return set_err(BM_ERR_INVALID, "an area of this batch was destroyed");
    if (!batch) return set_err(BM_ERR_INVALID, "null batch");
    batch->drain_profile();
    for (auto& p : batch->plan) {
        p.prof_n = 0;
        p.prof_ms = 0;
    }
    return BM_OK;
}

int bm_batch_launches_per_cycle(bm_batch batch, uint32_t* out) {
    if (batch && batch->detached) return set_err(BM_ERR_INVALID, "an area of this batch was destroyed");
    if (!batch || !out) return set_err(BM_ERR_INVALID, "null argument");
    uint32_t n = (batch->intake_blocks ? 1u : 0u) + 1u;   // copies, cycle end
    n += batch->plan_launches;
    *out = n;
    return BM_OK;
}

int bm_batch_device_errors(bm_batch batch, uint32_t* bits) {
    if (batch && batch->detached) return set_err(BM_ERR_INVALID, "an area of this batch was destroyed");
    if (!batch || !bits) return set_err(BM_ERR_INVALID, "null argument");
    uint32_t all = 0;
    for (bm_area A : batch->areas) {
        uint32_t b = 0;
        int rc = bm_area_device_errors(A, &b);
        if (rc != BM_OK && rc != BM_ERR_TIMEOUT) return rc;
        all |= b;
    }
    *bits = all;
    if (all) return set_err(BM_ERR_TIMEOUT, "device-side wait timed out in a batched area (error bits 0x%x)", all);
    return BM_OK;
}

int bm_batch_autotune(bm_batch batch, const char* cache_path, uint32_t* n_tuned) {
    if (batch && batch->detached) return set_err(BM_ERR_INVALID, "an area of this batch was destroyed");
    if (!batch) return set_err(BM_ERR_INVALID, "null batch");
    bm_batch_s* B = batch;
    DevGuard g(B->ctx->device);
    cudaStream_t s = B->stream();
    std::map<std::string, Tuned> cache = read_cache(cache_path);
    uint32_t tuned = 0;
    static const uint32_t kTargets[] = {4096, 8192, 16384, 32768, 65536, 131072};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // Device milliseconds of 5 launches of the step as planned (one warm-up
    // launch first).
    auto time_step = [&](const bm_batch_s::StepPlan& p) {
        launch_fused_batch(p.fb, s);
        cudaEventRecord(e0, s);
        for (int r = 0; r < 5; r++) launch_fused_batch(p.fb, s);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms;
    };
    for (auto& p : B->plan) {
        if (p.form != bm_batch_s::F_FUSED) continue;
        const std::string key = step_key(p);
        auto hit = cache.find(key);
        if (hit != cache.end()) {
            p.shape = {hit->second.stages, hit->second.ctas};
            if (!apply_target(B, p, hit->second.target, hit->second.staged != 0)) {
                p.shape = {};
                build_fused(p);
            }
            tuned++;
            continue;
        }
        // Save what the trials overwrite.
        std::vector<Range> ranges;
        for (auto& [A, t] : p.tufts) step_ranges(A, p.st.layer, t, (p.st.arg & 1) != 0, ranges);
        uint64_t total = 0;
        for (auto& r : ranges) total += r.n;
        uint8_t* save = nullptr;
        if (cudaMalloc(&save, total) != cudaSuccess) {
            cudaGetLastError();
            continue;   // not enough memory to tune this step safely: keep its tiles
        }
        uint64_t o = 0;
        for (auto& r : ranges) { cudaMemcpyAsync(save + o, r.p, r.n, cudaMemcpyDeviceToDevice, s); o += r.n; }
        // The tile size and footprint form first, with the default shape; then
        // the ring depth and CTAs per SM for the chosen tiles (shapes that
        // plan the same launches as one already timed are not timed again).
        Tuned best;
        float best_ms = 1e30f;
        p.shape = {};
        for (uint32_t staged : {0u, 1u}) {
            for (uint32_t target : kTargets) {
                if (!apply_target(B, p, target, staged != 0)) continue;
                const float ms = time_step(p);
                if (ms < best_ms) {
                    best_ms = ms;
                    best.target = target;
                    best.staged = staged;
                }
            }
        }
        if (best.target) {
            std::vector<std::pair<std::vector<uint32_t>, std::vector<uint32_t>>> seen;
            for (uint32_t stages : {0u, 2u, 3u}) {
                for (uint32_t ctas : {0u, 1u, 2u}) {
                    p.shape = {stages, ctas};
                    if (!apply_target(B, p, best.target, best.staged != 0)) continue;
                    std::vector<uint32_t> nst;
                    for (void* q : p.fb.params) nst.push_back(fused_batch_stages(q));
                    auto sig = std::make_pair(p.fb.grids, p.fb.smems);
                    sig.second.insert(sig.second.end(), nst.begin(), nst.end());
                    if (std::find(seen.begin(), seen.end(), sig) != seen.end()) continue;
                    seen.push_back(sig);
                    const float ms = (stages == 0 && ctas == 0) ? best_ms : time_step(p);
                    if (ms < best_ms * 0.98f) {
                        best_ms = ms;
                        best.stages = stages;
                        best.ctas = ctas;
                    }
                }
            }
        }
        p.shape = {best.stages, best.ctas};
        if (best.target == 0 || !apply_target(B, p, best.target, best.staged != 0)) {
            p.shape = {};
            build_fused(p);
        }
        o = 0;
        for (auto& r : ranges) { cudaMemcpyAsync(r.p, save + o, r.n, cudaMemcpyDeviceToDevice, s); o += r.n; }
        cudaStreamSynchronize(s);
        cudaFree(save);
        if (best.target) { cache[key] = best; tuned++; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    count_launches(B);
    B->drop_graph();
    write_cache(cache_path, cache);
    if (n_tuned) *n_tuned = tuned;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_err(e, "bm_batch_autotune");
    return BM_OK;
}

}  // extern "C"
