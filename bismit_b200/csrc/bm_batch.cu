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
// A project-written autotuner (bm_batch_autotune) picks the tile size of each
// batched tuft step by timing candidates on the live batch (with the touched
// buffers saved and restored) and can keep its choices in a cache file.
#include <cstdio>
#include <cstring>
#include <map>
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
    uint32_t x;         // tuft or control index
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

// Sub-stages of an unfused tuft, batched like the per-cell steps (item =
// synapse, synapse, dendrite, cell).
constexpr int BK_FLAGS = 100, BK_SYN = 101, BK_DEN = 102, BK_TFT = 103;

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
__global__ void __launch_bounds__(kCellBlock) k_batch_cells(const CellJob* __restrict__ jobs, uint32_t n_jobs) {
    const CellJob& J = jobs[block_job(jobs, n_jobs)];
    const uint32_t i = (blockIdx.x - J.block0) * kCellBlock + threadIdx.x;
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
    case BK_FLAGS: {
        // tft_set_syn_flags, cl/syns.cl:23-33, for the tuft's synapses.
        const uint64_t si = J.L.tft[J.x].syn_idz + i;
        uint8_t* fl = J.L.buf[BM_BUF_SYN_FLAG_SETS];
        fl[si] = (uint8_t)((fl[si] & ~kSynPrevActiveFlag) | (J.L.buf[BM_BUF_SYN_STATES][si] ? kSynPrevActiveFlag : 0));
        break;
    }
    case BK_SYN: syn_cycle_item(J.axns, J.slices, J.L, J.x, i); break;
    case BK_DEN: den_cycle_item(J.L, J.x, rnd_at(J.L.tft[J.x].rnd_key_den, J.ctl->cycle), i); break;
    case BK_TFT: tft_cycle_item(J.L, J.x, i); break;
    default: break;
    }
}

__global__ void __launch_bounds__(kIntakeBlock)
    k_batch_intake(const IntakeJob* __restrict__ jobs, uint32_t n_jobs, const BatchCtl* __restrict__ bc) {
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
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) ctls[i]->cycle += 1;
    if (i == 0) bc->cursor += 1;
}

__global__ void k_batch_begin(BatchCtl* bc, const uint8_t* frames, uint64_t frame_bytes) {
    bc->frames = frames;
    bc->cursor = 0;
    bc->frame_bytes = frame_bytes;
}

// Per-cell step kind -> launch.
void launch_cells(int st, const CellJob* jobs, uint32_t n_jobs, uint32_t n_blocks, cudaStream_t s) {
    if (!n_blocks) return;
    switch (st) {
#define BM_CELLS(K) \
    case K: k_batch_cells<K><<<n_blocks, kCellBlock, 0, s>>>(jobs, n_jobs); break;
        BM_CELLS(ST_SSC_CYCLE)
        BM_CELLS(ST_INHIB_SIMPLE)
        BM_CELLS(ST_INHIB_PASS)
        BM_CELLS(ST_PYR_OUTPUT)
        BM_CELLS(ST_INTRA_COL)
        BM_CELLS(ST_PYR_CYCLE)
        BM_CELLS(ST_DST_MTP)
        BM_CELLS(ST_SSC_MTP)
        BM_CELLS(BK_FLAGS)
        BM_CELLS(BK_SYN)
        BM_CELLS(BK_DEN)
        BM_CELLS(BK_TFT)
#undef BM_CELLS
    default: break;
    }
}

bool is_cell_step(int st) {
    return st == ST_SSC_CYCLE || st == ST_INHIB_SIMPLE || st == ST_INHIB_PASS || st == ST_PYR_OUTPUT ||
           st == ST_INTRA_COL || st == ST_PYR_CYCLE || st == ST_DST_MTP || st == ST_SSC_MTP;
}

}  // namespace

struct bm_batch_s {
    enum Form { F_CELLS, F_FUSED, F_EACH, F_END };
    struct CellLaunch {
        int kind;
        CellJob* d_jobs;
        uint32_t n_jobs, n_blocks;
    };
    struct StepPlan {
        Step st;
        Form form = F_EACH;
        std::vector<CellLaunch> cells;   // F_CELLS: launches in order
        FusedBatch fb;
    };
    // Areas with one stage program, batched step by step.
    struct Group {
        std::vector<bm_area> areas;
        std::vector<StepPlan> plan;
        uint32_t launches = 0;
    };
    bm_ctx ctx = nullptr;
    std::vector<bm_area> areas;          // every area, in batch order
    std::vector<Group> groups;
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

namespace {

void free_plan(bm_batch_s::Group& G) {
    for (auto& p : G.plan) {
        for (auto& c : p.cells) cudaFree(c.d_jobs);
        free_fused_batch(p.fb);
    }
    G.plan.clear();
}

void free_batch(bm_batch_s* B) {
    if (!B) return;
    DevGuard g(B->ctx->device);
    B->drop_graph();
    for (auto& G : B->groups) free_plan(G);
    if (B->d_intake) cudaFree(B->d_intake);
    if (B->d_bctl) cudaFree(B->d_bctl);
    if (B->d_ctls) cudaFree(B->d_ctls);
    if (B->cap) cudaStreamDestroy(B->cap);
    delete B;
}

// Work items of a per-cell launch of kind k for step st of area A.
uint64_t items_of(const bm_area_s* A, int k, const Step& st) {
    const bm_layer_plan& L = A->plan.layers[st.layer];
    switch (k) {
    case ST_INTRA_COL: return (uint64_t)L.v_size * L.u_size;
    case BK_FLAGS:
    case BK_SYN: return (uint64_t)L.cells * L.tufts[st.idx].syns_per_tft;
    case BK_DEN: return (uint64_t)L.cells * L.tufts[st.idx].dens_per_tft;
    default: return L.cells;
    }
}

// One batched per-cell launch of kind k for step st over every area.
int add_cells(bm_batch_s::Group& G, bm_batch_s::StepPlan& p, int k) {
    const Step& st = p.st;
    std::vector<CellJob> jobs;
    uint64_t blocks = 0;
    for (bm_area A : G.areas) {
        CellJob J;
        std::memset(&J, 0, sizeof J);
        J.L = A->dl[st.layer];
        J.axns = A->axns();
        J.slices = A->slices;
        J.ctl = A->ctl;
        J.x = st.idx;
        if (k == ST_INHIB_SIMPLE) {
            J.key = A->inhib_key[st.layer][st.idx];
            J.radius = (int32_t)A->plan.layers[st.layer].ctrl[st.idx].field_radius;
        }
        const uint64_t n = items_of(A, k, st);
        if (n > 0xFFFFFFFFull) return set_err(BM_ERR_UNSUPPORTED, "batched step of more than 2^32 items");
        J.n = (uint32_t)n;
        J.block0 = (uint32_t)blocks;
        blocks += (n + kCellBlock - 1) / kCellBlock;
        jobs.push_back(J);
    }
    if (blocks > 0x7FFFFFFFull) return set_err(BM_ERR_UNSUPPORTED, "batched step of too many blocks");
    bm_batch_s::CellLaunch c{k, nullptr, (uint32_t)jobs.size(), (uint32_t)blocks};
    cudaError_t e = cudaMalloc(&c.d_jobs, jobs.size() * sizeof(CellJob));
    if (e == cudaSuccess) e = cudaMemcpy(c.d_jobs, jobs.data(), jobs.size() * sizeof(CellJob), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        if (c.d_jobs) cudaFree(c.d_jobs);
        return cuda_err(e, "batched step jobs");
    }
    p.cells.push_back(c);
    p.form = bm_batch_s::F_CELLS;
    return BM_OK;
}

int build_fused(bm_batch_s::Group& G, bm_batch_s::StepPlan& p) {
    std::vector<FusedJob> jobs;
    for (bm_area A : G.areas) {
        if (!A->fused.t[p.st.layer][p.st.idx].ok) return BM_OK;
        jobs.push_back({&A->fused, &A->dl[p.st.layer], A->axns(), A->slices, A->ctl});
    }
    int rc = prepare_fused_batch(p.fb, jobs, p.st.layer, p.st.idx);
    if (rc != BM_OK) return rc;
    p.form = p.fb.ok ? bm_batch_s::F_FUSED : bm_batch_s::F_EACH;
    return BM_OK;
}

int build_step(bm_batch_s::Group& G, bm_batch_s::StepPlan& p) {
    const Step& st = p.st;
    if (st.kind == ST_CYCLE_END) {
        p.form = bm_batch_s::F_END;
        return BM_OK;
    }
    if (is_cell_step(st.kind)) return add_cells(G, p, st.kind);
    if (st.kind != ST_TUFT) return BM_OK;   // the plain form's whole-layer tuft stages: each area's own
    bool none_ok = true, all_ok = true;
    for (bm_area A : G.areas) {
        const bool ok = A->fused.t[st.layer][st.idx].ok;
        none_ok = none_ok && !ok;
        all_ok = all_ok && ok;
    }
    if (all_ok) return build_fused(G, p);
    if (!none_ok) return BM_OK;
    // No area can take the fused kernel here (e.g. one-synapse dendrites):
    // the tuft's four stages, each batched.
    int rc = add_cells(G, p, BK_FLAGS);
    if (rc == BM_OK) rc = add_cells(G, p, BK_SYN);
    if (rc == BM_OK) rc = add_cells(G, p, BK_DEN);
    if (rc == BM_OK && G.areas[0]->plan.layers[st.layer].kind == BM_LYR_PYRAMIDAL) rc = add_cells(G, p, BK_TFT);
    return rc;
}

void count_launches(bm_batch_s::Group& G) {
    G.launches = 0;
    for (const auto& p : G.plan) {
        const Step& st = p.st;
        if (p.form == bm_batch_s::F_EACH) {
            // Each area's own launches for this step.
            for (bm_area A : G.areas) {
                const bm_layer_plan& L = A->plan.layers[st.layer];
                uint32_t per = 1;
                if (st.kind == ST_TUFT && !A->fused.t[st.layer][st.idx].ok) per = L.kind == BM_LYR_PYRAMIDAL ? 4 : 3;
                if (st.kind == ST_TUFTS_PLAIN) per = 1 + 2 * L.n_tufts + (L.kind == BM_LYR_PYRAMIDAL ? L.n_tufts : 0);
                G.launches += per;
            }
        } else if (p.form == bm_batch_s::F_CELLS) {
            G.launches += (uint32_t)p.cells.size();
        } else if (p.form == bm_batch_s::F_FUSED) {
            G.launches += 1;
        }
    }
}

// The group's steps; the cycle-end step is done once for the whole batch.
int build_plan(bm_batch_s::Group& G) {
    free_plan(G);
    for (const Step& st : G.areas[0]->steps) {
        bm_batch_s::StepPlan p;
        p.st = st;
        int rc = build_step(G, p);
        G.plan.push_back(p);
        if (rc != BM_OK) return rc;
    }
    count_launches(G);
    return BM_OK;
}

// The head-of-cycle copies: every tract, then every input of every area that
// no tract feeds, taken from the frame block in (area, input) order.
int build_intake(bm_batch_s* B) {
    if (B->d_intake) cudaFree(B->d_intake);
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
    for (const auto& T : B->tracts) {
        bm_area S = B->areas[T.src_area], D = B->areas[T.dst_area];
        IntakeJob J{};
        J.dst = D->axns() + D->plan.inputs[T.dst_input].axn_idz + T.dst_off;
        J.src = S->axns() + S->plan.outputs[T.src_output].axn_idz;
        J.len = S->plan.outputs[T.src_output].len;
        add(J);
    }
    for (uint32_t a = 0; a < B->areas.size(); a++) {
        bm_area A = B->areas[a];
        for (uint32_t i = 0; i < A->plan.n_inputs; i++) {
            bool fed = false;
            for (const auto& T : B->tracts) fed = fed || (T.dst_area == a && T.dst_input == i);
            if (fed) continue;
            IntakeJob J{};
            J.dst = A->axns() + A->plan.inputs[i].axn_idz;
            J.src_off = B->frame_bytes;
            J.len = A->plan.inputs[i].len;
            B->frame_bytes += J.len;
            add(J);
        }
    }
    if (jobs.empty()) return BM_OK;
    if (blocks > 0x7FFFFFFFull) return set_err(BM_ERR_UNSUPPORTED, "batched intake too large");
    cudaError_t e = cudaMalloc(&B->d_intake, jobs.size() * sizeof(IntakeJob));
    if (e == cudaSuccess) e = cudaMemcpy(B->d_intake, jobs.data(), jobs.size() * sizeof(IntakeJob), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_err(e, "batched intake jobs");
    B->n_intake = (uint32_t)jobs.size();
    B->intake_blocks = (uint32_t)blocks;
    return BM_OK;
}

void enqueue_batch_cycle(bm_batch_s* B, cudaStream_t s) {
    if (B->intake_blocks)
        k_batch_intake<<<B->intake_blocks, kIntakeBlock, 0, s>>>(B->d_intake, B->n_intake, B->d_bctl);
    for (auto& G : B->groups)
        for (auto& p : G.plan) {
            switch (p.form) {
            case bm_batch_s::F_CELLS:
                for (auto& c : p.cells) launch_cells(c.kind, c.d_jobs, c.n_jobs, c.n_blocks, s);
                break;
            case bm_batch_s::F_FUSED: launch_fused_batch(p.fb, s); break;
            case bm_batch_s::F_END: break;
            default:
                for (bm_area A : G.areas) exec_step(A, p.st, s);
                break;
            }
        }
    const uint32_t n = (uint32_t)B->areas.size();
    k_batch_cycle_end<<<(n + 127) / 128, 128, 0, s>>>(B->d_ctls, n, B->d_bctl);
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

int run_cycles(bm_batch_s* B, const void* frames, uint32_t n_cycles) {
    cudaStream_t s = B->stream();
    for (bm_area A : B->areas) run_pending_verifies(A, s);
    k_batch_begin<<<1, 1, 0, s>>>(B->d_bctl, (const uint8_t*)frames, B->frame_bytes);
    if (B->use_graph) {
        int rc = ensure_graph(B);
        if (rc != BM_OK) return rc;
        for (uint32_t k = 0; k < n_cycles; k++) {
            cudaError_t e = cudaGraphLaunch(B->exec, s);
            if (e != cudaSuccess) return cuda_err(e, "cudaGraphLaunch");
        }
    } else {
        for (uint32_t k = 0; k < n_cycles; k++) enqueue_batch_cycle(B, s);
    }
    for (bm_area A : B->areas) A->host_cycle += n_cycles;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_err(e, "batched cycle");
    return BM_OK;
}

// --------------------------------------------------------- autotuner -----
// The buffers one tuft step writes, per area: synapse states and flags,
// dendrite raw states, states and activities, and (pyramidal) the eight
// cell-tuft buffers.
struct Range {
    uint8_t* p;
    uint64_t n;
};
void step_ranges(bm_area_s* A, uint32_t i, uint32_t t, std::vector<Range>& out) {
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
}

std::string step_key(bm_batch_s::Group& G, const Step& st) {
    std::string k = "L" + std::to_string(st.layer) + "T" + std::to_string(st.idx);
    for (bm_area A : G.areas) {
        const bm_layer_plan& L = A->plan.layers[st.layer];
        const bm_tuft_plan& T = L.tufts[st.idx];
        char buf[96];
        snprintf(buf, sizeof buf, ":%ux%ux%u/%u/%u/%u", L.v_size, L.u_size, L.depth, T.syns_per_tft,
                 T.syns_per_den, T.n_src_uniq);
        k += buf;
    }
    return k;
}

std::map<std::string, uint32_t> read_cache(const char* path) {
    std::map<std::string, uint32_t> m;
    if (!path) return m;
    FILE* f = fopen(path, "r");
    if (!f) return m;
    char key[4096];
    unsigned v;
    while (fscanf(f, "%4095s %u", key, &v) == 2) m[key] = v;
    fclose(f);
    return m;
}

void write_cache(const char* path, const std::map<std::string, uint32_t>& m) {
    if (!path) return;
    FILE* f = fopen(path, "w");
    if (!f) return;
    for (auto& kv : m) fprintf(f, "%s %u\n", kv.first.c_str(), kv.second);
    fclose(f);
}

// Retiles tuft (i, t) of every area for `target` synapses per tile and
// rebuilds the step's batched launch. False when some area cannot take it.
bool apply_target(bm_batch_s* B, bm_batch_s::Group& G, bm_batch_s::StepPlan& p, uint32_t target) {
    for (bm_area A : G.areas)
        if (!retile_fused_tuft(A->fused, A->plan, p.st.layer, p.st.idx, target)) return false;
    for (bm_area A : G.areas) {
        A->verify_pending[p.st.layer] = true;
        run_pending_verifies(A, B->stream());
    }
    return build_fused(G, p) == BM_OK && p.form == bm_batch_s::F_FUSED;
}

}  // namespace

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
    B->areas.assign(areas, areas + n_areas);
    cudaError_t e = cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) { free_batch(B); return cuda_err(e, "cudaStreamCreate"); }

    std::vector<AreaCtl*> ctls;
    for (bm_area A : B->areas) ctls.push_back(A->ctl);
    e = cudaMalloc(&B->d_bctl, sizeof(BatchCtl));
    if (e == cudaSuccess) e = cudaMemset(B->d_bctl, 0, sizeof(BatchCtl));
    if (e == cudaSuccess) e = cudaMalloc(&B->d_ctls, ctls.size() * sizeof(AreaCtl*));
    if (e == cudaSuccess) e = cudaMemcpy(B->d_ctls, ctls.data(), ctls.size() * sizeof(AreaCtl*), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { free_batch(B); return cuda_err(e, "batch set-up"); }
    // Areas with equal stage programs form one group (first appearance order).
    for (bm_area A : B->areas) {
        bm_batch_s::Group* G = nullptr;
        for (auto& g2 : B->groups)
            if (g2.areas[0]->steps == A->steps) G = &g2;
        if (!G) {
            B->groups.emplace_back();
            G = &B->groups.back();
        }
        G->areas.push_back(A);
    }
    int rc = build_intake(B);
    for (auto& G : B->groups)
        if (rc == BM_OK) rc = build_plan(G);
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
    if (!batch || !out) return set_err(BM_ERR_INVALID, "null argument");
    *out = batch->frame_bytes;
    return BM_OK;
}

int bm_batch_connect(bm_batch batch, uint32_t src_area, uint32_t src_output, uint32_t dst_area, uint32_t dst_input,
                     uint64_t dst_offset) {
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
    return BM_OK;
}

int bm_batch_cycle_frames_device(bm_batch batch, const void* dev_frames, uint32_t n_cycles) {
    if (!batch || !dev_frames) return set_err(BM_ERR_INVALID, "null argument");
    if (!batch->frame_bytes) return set_err(BM_ERR_INVALID, "the batch has no input that a tract does not feed");
    DevGuard g(batch->ctx->device);
    return run_cycles(batch, dev_frames, n_cycles);
}

int bm_batch_launches_per_cycle(bm_batch batch, uint32_t* out) {
    if (!batch || !out) return set_err(BM_ERR_INVALID, "null argument");
    uint32_t n = (batch->intake_blocks ? 1u : 0u) + 1u;   // copies, cycle end
    for (const auto& G : batch->groups) n += G.launches;
    *out = n;
    return BM_OK;
}

int bm_batch_device_errors(bm_batch batch, uint32_t* bits) {
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
    if (!batch) return set_err(BM_ERR_INVALID, "null batch");
    bm_batch_s* B = batch;
    DevGuard g(B->ctx->device);
    cudaStream_t s = B->stream();
    std::map<std::string, uint32_t> cache = read_cache(cache_path);
    uint32_t tuned = 0;
    static const uint32_t kTargets[] = {4096, 8192, 16384, 32768, 65536};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (auto& G : B->groups)
    for (auto& p : G.plan) {
        if (p.form != bm_batch_s::F_FUSED) continue;
        const std::string key = step_key(G, p.st);
        auto hit = cache.find(key);
        if (hit != cache.end()) {
            if (!apply_target(B, G, p, hit->second)) build_fused(G, p);
            tuned++;
            continue;
        }
        // Save what the trials overwrite.
        std::vector<Range> ranges;
        for (bm_area A : G.areas) step_ranges(A, p.st.layer, p.st.idx, ranges);
        uint64_t total = 0;
        for (auto& r : ranges) total += r.n;
        uint8_t* save = nullptr;
        if (cudaMalloc(&save, total) != cudaSuccess) {
            cudaGetLastError();
            continue;   // not enough memory to tune this step safely: keep its tiles
        }
        uint64_t o = 0;
        for (auto& r : ranges) { cudaMemcpyAsync(save + o, r.p, r.n, cudaMemcpyDeviceToDevice, s); o += r.n; }
        uint32_t best_t = 0;
        float best_ms = 1e30f;
        for (uint32_t target : kTargets) {
            if (!apply_target(B, G, p, target)) continue;
            launch_fused_batch(p.fb, s);   // warm-up
            cudaEventRecord(e0, s);
            for (int r = 0; r < 5; r++) launch_fused_batch(p.fb, s);
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best_ms) { best_ms = ms; best_t = target; }
        }
        if (best_t == 0 || !apply_target(B, G, p, best_t)) build_fused(G, p);
        o = 0;
        for (auto& r : ranges) { cudaMemcpyAsync(r.p, save + o, r.n, cudaMemcpyDeviceToDevice, s); o += r.n; }
        cudaStreamSynchronize(s);
        cudaFree(save);
        if (best_t) { cache[key] = best_t; tuned++; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (auto& G : B->groups) count_launches(G);
    B->drop_graph();
    write_cache(cache_path, cache);
    if (n_tuned) *n_tuned = tuned;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_err(e, "bm_batch_autotune");
    return BM_OK;
}

}  // extern "C"
