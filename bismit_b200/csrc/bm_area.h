// bm_area.h -- the library's internal view of contexts and areas, and the
// per-area stage program (the ordered steps of one cycle) that the one-area
// path and the batched path (bm_batch.cu) both execute.
#pragma once
#include <atomic>
#include <bitset>
#include <cstdint>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "bm_fused.h"
#include "bm_kernels.h"

namespace bm {

// Kernel kinds for per-launch timing.
enum Kind {
    K_SYN_FLAGS, K_SYN_CYCLE, K_DEN_CYCLE, K_TFT_CYCLE, K_SSC_CYCLE, K_INHIB_SIMPLE, K_INHIB_PASS,
    K_SSC_MTP, K_PYR_CYCLE, K_PYR_OUTPUT, K_INTRA_COL, K_TFT_DST_MTP, K_CYCLE_END, K_INTAKE,
    K_FUSED_TUFT, K_TUFT_CELLS, K_INHIB_MTP, K_PYR_TAIL, K_REGROW, K_SMOOTH, K_RETINA, K_COUNT
};
const char* const kKindNames[K_COUNT] = {
    "tft_set_syn_flags", "syn_cycle", "den_cycle_tft", "tft_cycle", "ssc_cycle", "inhib_simple",
    "inhib_passthrough", "ssc_mtp_simple", "pyr_cycle", "pyr_output", "inhib_intra_column", "tft_dst_mtp",
    "cycle_end", "intake", "fused_tuft_cycle", "tuft_cells", "inhib_mtp", "pyr_tail", "regrow",
    "smooth_activity", "retina"};

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DevGuard() {
        int cur;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// One step of an area's cycle. Areas with equal step lists can be cycled
// together, one batched launch per step (bm_batch.cu).
enum StepKind : uint8_t {
    ST_TUFT,          // tuft `idx` of layer `layer`: fused launch, or its four plain stages
    ST_TUFTS_PLAIN,   // plain form: flags of the layer, then each stage per tuft
    ST_SSC_CYCLE,
    ST_INHIB_SIMPLE,  // control `idx` hosted on `layer`
    ST_INHIB_PASS,
    ST_PYR_OUTPUT,
    ST_INTRA_COL,
    ST_PYR_CYCLE,
    ST_DST_MTP,       // distal learning of tuft `idx`
    ST_SSC_MTP,
    ST_CYCLE_END,
    // Fused forms (the fused execution path, layers with plain slices):
    ST_INHIB_MTP,     // ST_INHIB_SIMPLE `idx` followed by ST_SSC_MTP (arg 1) of the same layer
    ST_PYR_TAIL,      // ST_PYR_CYCLE, control `idx` (intra-column or output; 0xFF none), and
                      // (arg 1) ST_DST_MTP of every distal tuft, in that order
    ST_REGROW,        // regrowth of every tuft of every data layer (acts on its cycles only)
    ST_SMOOTH,        // activity smoother `idx` hosted on `layer` (six lattice launches)
    ST_FILTER,        // input filter chain `idx`, from its first buffer to its target slices
};
struct Step {
    uint8_t kind, layer, idx, arg;
    uint8_t tufts = 0;   // ST_PYR_TAIL: per-cell tufts (bit t) it runs first, folded in
    bool operator==(const Step& o) const {
        return kind == o.kind && layer == o.layer && idx == o.idx && arg == o.arg && tufts == o.tufts;
    }
};

// What a step of one area reads and writes, at the granularity its kernels
// touch: axon slices, the synapse / dendrite / cell-tuft arrays of one tuft of
// a layer, and the cell arrays of a layer. Two steps of an area whose accesses
// do not conflict may run concurrently.
struct StepAccess {
    std::bitset<BM_MAX_SLICES> ax_r, ax_w;
    uint64_t tf_r = 0, tf_w = 0;   // bit layer * BM_MAX_TUFTS + tuft
    uint32_t ce_r = 0, ce_w = 0;   // bit layer
    bool all = false;              // touches everything (regrowth, the cycle end)
    StepAccess& operator|=(const StepAccess& o) {
        ax_r |= o.ax_r; ax_w |= o.ax_w;
        tf_r |= o.tf_r; tf_w |= o.tf_w;
        ce_r |= o.ce_r; ce_w |= o.ce_w;
        all = all || o.all;
        return *this;
    }
};
inline bool conflict(const StepAccess& a, const StepAccess& b) {
    if (a.all || b.all) return true;
    if ((a.ax_w & (b.ax_r | b.ax_w)).any() || (b.ax_w & a.ax_r).any()) return true;
    if ((a.tf_w & (b.tf_r | b.tf_w)) || (b.tf_w & a.tf_r)) return true;
    if ((a.ce_w & (b.ce_r | b.ce_w)) || (b.ce_w & a.ce_r)) return true;
    return false;
}

}  // namespace bm

struct bm_ctx_s {
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t user = nullptr;
    bool user_set = false;
    // References: the caller's handle (until bm_ctx_destroy) plus one per
    // live area, batch, server and writer made on it; the last release frees
    // the context, so destroying it before its children is safe.
    std::atomic<int> refs{1};
    // Device memory of the areas and batches made on this context comes from
    // this pool in stream order when set (a server's contexts: areas come and
    // go beside the ticks, and a plain free would wait for the whole device).
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream() const { return user_set ? user : own; }
};
namespace bm {
// A non-blocking stream at `base`'s priority: a side or capture stream runs
// its share of a cycle at the priority of the stream it forks from.
inline cudaError_t stream_like(cudaStream_t base, cudaStream_t* out) {
    int prio = 0;
    if (cudaStreamGetPriority(base, &prio) != cudaSuccess) {
        cudaGetLastError();
        prio = 0;
    }
    return cudaStreamCreateWithPriority(out, cudaStreamNonBlocking, prio);
}
// A device allocation of an object made on context c: from c's pool in
// stream order on c's stream when it has one, else cudaMalloc.
inline cudaError_t dev_alloc(bm_ctx c, void** p, size_t n) {
    if (c && c->pool) return cudaMallocFromPoolAsync(p, n, c->pool, c->stream());
    return cudaMalloc(p, n);
}
template <class T> inline cudaError_t dev_alloc(bm_ctx c, T** p, size_t n) {
    return dev_alloc(c, (void**)p, n);
}
// Frees what dev_alloc gave: in stream order on s when it came from a pool,
// else cudaFree (which first waits for the device).
inline void dev_free(void* p, bool pooled, cudaStream_t s) {
    if (!p) return;
    if (pooled) cudaFreeAsync(p, s);
    else cudaFree(p);
}
// A host-mapped word the device writes and the host polls (an area's error
// mirror): slots of page-locked blocks kept for the process, so areas that
// come and go page-lock and release nothing.
cudaError_t host_word_get(unsigned int** host, unsigned int** dev);
void host_word_put(unsigned int* host);
inline void ctx_retain(bm_ctx c) {
    if (c) c->refs.fetch_add(1, std::memory_order_relaxed);
}
void ctx_release(bm_ctx c);   // frees the context with its last reference
}  // namespace bm

struct bm_area_s {
    using Step = bm::Step;
    bm_ctx ctx = nullptr;
    bm_area_plan plan;
    uint8_t* slab = nullptr;
    bm::AreaCtl* ctl = nullptr;
    unsigned int* host_err = nullptr;   // host-mapped mirror of ctl->error (written when non-zero)
    bool pooled = false;                // device memory from the creating context's pool
    bm::SliceRec* slices = nullptr;
    bm::DevLayer dl[BM_MAX_LAYERS];
    uint64_t inhib_key[BM_MAX_LAYERS][BM_MAX_CTRL];
    uint64_t host_cycle = 0;
    bool verify_pending[BM_MAX_LAYERS] = {};   // sources or flags written since the last check
    uint32_t exec_path = BM_PATH_FUSED;
    bm::FusedArea fused;
    bool profiling = false;
    struct Rec { int kind; cudaEvent_t a, b; };
    std::vector<Rec> pending;
    std::vector<cudaEvent_t> pool;
    uint64_t prof_launches[bm::K_COUNT] = {};
    double prof_ms[bm::K_COUNT] = {};
    uint32_t launches = 0;   // kernel launches of the last enqueued cycle
    std::vector<Step> steps; // the cycle's stage program
    bool end_in_tail = false;  // the last pyramidal tail also ends the cycle (no cycle-end launch)
    // Two-stream form of the program (schedule_area): steps on the side
    // stream, the side steps each main step waits for, events and the stream.
    std::vector<uint8_t> step_side;
    std::vector<std::vector<size_t>> step_waits;
    size_t last_side = SIZE_MAX;
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr;
    std::vector<cudaEvent_t> side_ev;
    // Front stream (schedule_area): the program's leading spatial-layer steps
    // (fused tuft, inhibition with learning) and the frame intake run there,
    // each ordered against the previous cycle only by what it touches, so a
    // cycle's spatial chain runs beside the previous cycle's pyramidal steps.
    // Their kernels take the cycle number from the host (the area's counter
    // advances at the end of the previous cycle on the main stream).
    size_t front_n = 0;                                  // leading steps on the front stream (0: none)
    std::vector<std::vector<size_t>> front_prev;         // per front step: steps of the previous cycle to wait for
    std::vector<std::vector<size_t>> front_waits;        // per later step: front steps of its cycle to wait for
    std::vector<size_t> intake_prev;                     // steps of the previous cycle the intake waits for
    std::vector<uint8_t> intake_readers;                 // later steps reading what the intake writes
    std::vector<uint8_t> main_ev_needed;                 // main steps a front step or the intake waits for
    std::bitset<BM_MAX_SLICES> front_ax_w;               // axon slices the front steps write
    std::vector<cudaEvent_t> front_ev, main_ev;
    cudaEvent_t intake_ev = nullptr;
    // Recorded on the main stream after work there that the front stream's
    // next steps must follow (verifications, batched cycles, tract copies,
    // control writes); the front stream waits for it at each cycle's start.
    cudaEvent_t main_mark = nullptr;
    cudaStream_t front = nullptr;
    bool front_last = false;      // the latest enqueued cycle used the front stream
    std::vector<bm_sampler_s*> samplers;   // per-cycle readback channels (bm_sampler.cu)
    // Host frames (bm_area_write_input) are copied into a pinned slot during
    // the call, uploaded on `up` into a device slot while earlier cycles
    // run, and moved into place on the area's stream. Two slots, each reused
    // once the area's stream has taken the frame it held (up_taken).
    cudaStream_t up = nullptr;
    uint8_t* up_host[2] = {};
    uint8_t* up_dev[2] = {};
    cudaEvent_t up_loaded[2] = {}, up_taken[2] = {};
    uint32_t up_next = 0;
    size_t up_cap = 0;
    // Samplers' device-to-host copies run on `down`, from a device copy of
    // the sampled range taken on the cycling stream.
    cudaStream_t down = nullptr;
    // Activity smoothers: group centers per (host layer, control), six
    // lattices in center_off ranges.
    int32_t* d_centers[BM_MAX_LAYERS][BM_MAX_CTRL] = {};
    uint32_t center_off[BM_MAX_LAYERS][BM_MAX_CTRL][7] = {};
    // Per data layer, bit t: tuft t may hold source slice ids outside its
    // pool (written by the caller), so its steps may read any axon slice.
    uint8_t foreign_src[BM_MAX_LAYERS] = {};
    uint32_t access_version = 0;   // bumped whenever foreign_src changes
    std::atomic<uint32_t> n_batches{0};   // batches holding this area (its tiles are retiled only when one does)
    std::vector<bm_batch_s*> batches;   // the batches holding it (detached when it is destroyed)
    // Regrowth (absent when disabled): one job per (data layer, tuft), layers
    // in cycle order, block0 counted within the area's own launch.
    std::vector<bm::RegrowJob> regrow;
    bm::RegrowJob* d_regrow = nullptr;
    uint32_t regrow_blocks = 0;
    int8_t* grow_offs = nullptr;             // the growth offset pools (v then u)
    bm::TuftGeo* d_geo = nullptr;            // per (layer, tuft): layer * BM_MAX_TUFTS + tuft
    bm::TuftGeo geo[BM_MAX_LAYERS][BM_MAX_TUFTS] = {};

    cudaStream_t stream() const { return ctx->stream(); }
    // Front stream in use this cycle (see front_n).
    bool front_active() const;
    // The stream frame intakes go to: the front stream when it is in use.
    cudaStream_t intake_stream() const { return front_active() ? front : stream(); }
    // Marks the main stream's current position for the front stream.
    void mark_main() {
        if (main_mark) cudaEventRecord(main_mark, stream());
    }
    // Device error bits a completed cycle mirrored to the host (0: none seen).
    unsigned int seen_errors() const { return host_err ? *(volatile const unsigned int*)host_err : 0u; }
    uint8_t* axns() const { return slab + plan.axon_off; }

    cudaEvent_t ev() {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    // Every stage launch sits in an NVTX range named after its kernel kind
    // (a no-op unless a profiler is attached), and is timed with CUDA events
    // when profiling is on.
    template <class F> void run(int kind, F&& f) {
        if (kind != bm::K_INTAKE) launches++;
        struct Range {
            explicit Range(const char* n) { nvtxRangePushA(n); }
            ~Range() { nvtxRangePop(); }
        } range(bm::kKindNames[kind]);
        if (!profiling) { f(); return; }
        Rec r{kind, ev(), ev()};
        cudaEventRecord(r.a, stream());
        f();
        cudaEventRecord(r.b, stream());
        pending.push_back(r);
    }
    void drain_profile() {
        for (auto& r : pending) {
            float ms = 0.f;
            cudaEventSynchronize(r.b);
            cudaEventElapsedTime(&ms, r.a, r.b);
            prof_launches[r.kind]++;
            prof_ms[r.kind] += ms;
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        pending.clear();
    }
};


namespace bm {

// The steps of one cycle of A (CorticalArea::cycle order).
// `fold_cell_tufts`: per-cell tuft steps of a pyramidal layer fold into its
// tail (one launch fewer; worth it while that work is small, see
// kFoldCellTufts), else they stay steps of their own.
void area_steps(const bm_area_s* A, std::vector<Step>& out, bool fold_cell_tufts);
// Cells of the pyramidal layers with per-cell (unfused) tufts: up to this many
// (over an area, or over a batch's areas) those tufts fold into the tail.
// Beyond it they stay a step of their own, which overlaps a side-stream tuft
// step where the tail, after the streams join, would not.
constexpr uint64_t kFoldCellTufts = 16384;
uint64_t cell_tuft_cells(const bm_area_s* A);
// Enqueues one step of A on stream s (a pyramidal tail with end_cycle also
// ends the cycle).
void exec_step(bm_area_s* A, const Step& st, cudaStream_t s, bool end_cycle = false);
// Recompiles the gather offsets of layers whose sources or flags were written.
void run_pending_verifies(bm_area_s* A, cudaStream_t s);
// Rebuilds A->geo (the tiled tufts' footprint geometry that regrowth uses).
void refresh_geo(bm_area_s* A);
// The accesses of step st of A; for a tuft step, of tuft `t` (the step's own
// tuft unless given).
StepAccess step_access(const bm_area_s* A, const Step& st, int t = -1);
// Input filter chains run when A has some and BM_SET_BYPASS_FILTERS is off.
inline bool filters_run(const bm_area_plan& P) {
    return P.n_filter_chains && !(P.settings & BM_SET_BYPASS_FILTERS);
}
// Where bytes [off, off + len) of input `input`'s frame land: piece k takes
// bytes off + pieces[k].off .. + pieces[k].len of the frame to pieces[k].dst,
// the input's axons, or, for a source whose filter chain runs, that chain's
// first buffer (the chain then writes the axons at the head of each cycle).
struct FramePiece {
    uint32_t off, len;
    uint8_t* dst;
};
void frame_pieces(bm_area_s* A, uint32_t input, uint32_t off, uint32_t len, std::vector<FramePiece>& out);
// Splits A's program over its stream and a side stream (see step_access).
int schedule_area(bm_area_s* A);
// Records caller-written source slice ids of layer i (see foreign_src).
void note_sources(bm_area_s* A, uint32_t i, uint64_t b, uint64_t e, const uint8_t* data, bool exact);
// After a cycle of A enqueued on stream s: sends each sampler's frame, or
// skips it, or waits for the receiver (bm_sampler.cu).
int sample_after_cycle(bm_area_s* A, cudaStream_t s);
// The slab range a sampler reads.
void sampler_range(const bm_sampler_s* S, uint64_t* off, uint64_t* len);
void free_samplers(bm_area_s* A);
// Detaches A from the batches holding it before it is destroyed (bm_batch.cu).
void detach_from_batches(bm_area_s* A);
// One batched cycle over device frames that does not refuse areas with
// device error bits: the caller (the server) checked them itself before
// taking frames from its queues (bm_batch.cu).
int batch_cycle_frames_unchecked(bm_batch_s* B, const void* dev_frames);
int cuda_err(cudaError_t e, const char* what);

}  // namespace bm
