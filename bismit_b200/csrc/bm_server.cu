// bm_server.cu -- serving: a continuous-batching loop over cortex sessions.
//
// A session is one area (an instance of a layer map) with a queue of input
// frames. Sessions are opened at any time and wait in a FIFO until the device
// memory budget has room for their state (the slab, the compiled gather
// offsets and the control blocks, known exactly from the resolved plan before
// anything is allocated). Admitted sessions keep their state resident until
// they are closed and drained.
//
// Every tick cycles each resident session that has a pending frame exactly
// once, all of them in one batch (bm_batch.cu: one launch per stage step per
// layer-map group, replayed from a CUDA graph); the batch is rebuilt only when
// the set of sessions in the tick changes. Frames of the tick are packed into
// one pinned block and copied in with one transfer; the sessions' output axons
// are gathered on the device and come back with one transfer. Ticks are
// pipelined two deep: a call queues tick N and then completes tick N - 1, so
// the host's packing and bookkeeping overlap the GPU's cycles (pinned blocks
// are double-buffered). While tick N runs the host also admits waiting
// sessions: their areas are built and grown on a second stream, so set-up
// overlaps the running cycles too.
//
// Admission runs off the tick path: a builder thread owned by the server
// builds and grows each admitted session's area on its own stream (and
// destroys retired ones), and a tick adopts the areas that are ready, so a
// tick never waits for a set-up or a teardown.
//
// Latency of a frame = completion of the tick that cycled it minus the moment
// it became ready (its submission, or the completion of the session's
// previous frame if that came later): admission waits show up in it.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "bm_area.h"

using namespace bm;

namespace {

using Clock = std::chrono::steady_clock;

double now_s() { return std::chrono::duration<double>(Clock::now().time_since_epoch()).count(); }

// Frames of one bm_server_submit call, consumed front to back.
struct Chunk {
    std::vector<uint8_t> bytes;
    uint32_t n = 0, next = 0;
    double submitted = 0;
};

// A session's frame queue: chunks in submission order.
struct FrameQueue {
    std::deque<Chunk> chunks;
    uint32_t len = 0;
    bool empty() const { return chunks.empty(); }
    const uint8_t* front() const { return chunks.front().bytes.data() + (size_t)chunks.front().next * len; }
    double front_submitted() const { return chunks.front().submitted; }
    void pop() {
        if (++chunks.front().next == chunks.front().n) chunks.pop_front();
    }
};

// One session's output in a tick's gathered output block.
struct OutJob {
    const uint8_t* src;
    uint64_t dst_off;
    uint32_t len;
    uint32_t block0;
};

constexpr uint32_t kGatherBlock = 256;

__global__ void __launch_bounds__(kGatherBlock) k_gather_outputs(const OutJob* __restrict__ jobs, uint32_t n_jobs,
                                                                 uint8_t* __restrict__ dst) {
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
    const OutJob& J = jobs[s_j];
    const uint32_t i = (blockIdx.x - J.block0) * kGatherBlock * 4 + threadIdx.x;
#pragma unroll
    for (uint32_t k = 0; k < 4; k++)
        if (i + k * kGatherBlock < J.len) dst[J.dst_off + i + k * kGatherBlock] = J.src[i + k * kGatherBlock];
}

}  // namespace

struct bm_server_s {
    struct Session {
        uint32_t id = 0;
        bm_area_desc desc;
        uint64_t seed = 0;
        uint64_t bytes = 0;          // device bytes while resident
        bm_area area = nullptr;
        FrameQueue frames;
        uint8_t* out = nullptr;      // output 0 after the latest cycled frame (host memory)
        uint32_t out_len = 0, in_len = 0;
        uint64_t done = 0;           // frames cycled
        uint32_t inflight = 0;       // queued ticks holding one of its frames
        double last_done = 0;        // completion time of the latest cycled frame
        double opened = 0, admitted = 0;
        bool closing = false, resident = false, retired = false;
        bool failed = false;         // dropped after its area ended a cycle with device error bits
        // Set-up by the builder thread: kWaiting until the budget admits the
        // session, kQueued while the builder has it, then kBuilt or kFailed.
        std::atomic<int> build{0};
        int build_rc = BM_OK;
        std::string build_msg;       // the builder's error message (error text is per thread)
    };
    static constexpr int kWaiting = 0, kQueued = 1, kBuilt = 2, kFailed = 3;
    // A queued tick: its sessions (with their frames' submission times), its
    // pinned blocks and completion event.
    struct Tick {
        bool live = false;
        std::vector<Session*> members;
        std::vector<double> submitted;
        double syn = 0, started = 0;
        uint32_t buf = 0;
        uint32_t what = 0;    // BM_TICK_* bits of what the queueing call also did
        uint64_t no = 0;      // tick number
        double enq0 = 0, enq1 = 0;   // host time around queueing its work
    };
    bm_ctx ctx = nullptr;            // the serving stream
    bm_ctx setup = nullptr;          // area construction, overlapping the ticks
    // Sessions' areas and the batches over them draw device memory from one
    // pool in stream order (set-up on `setup`, batches and adopted areas on
    // `serve`, a context on the serving stream): memory retired sessions
    // release is freed behind the ticks that used it and reused by new ones,
    // with no allocation or free that waits for the device beside the ticks.
    cudaMemPool_t pool = nullptr;
    bm_ctx serve = nullptr;
    uint64_t budget = 0, used = 0;
    uint32_t next_id = 1;
    std::vector<Session*> sessions;  // every open session, in open order
    std::vector<uint32_t> failed_ids;    // sessions dropped after a device error
    bm_batch batch = nullptr;
    std::vector<Session*> members;   // the batch's sessions, in batch order
    uint8_t* h_frames[2] = {};       // pinned frame blocks (double-buffered)
    uint8_t* d_frames = nullptr;
    uint64_t frames_cap = 0;
    uint8_t* h_out[2] = {};          // pinned gathered-output blocks
    uint8_t* d_out = nullptr;
    uint64_t out_cap = 0;
    OutJob* d_outjobs = nullptr;     // the current batch's output gather
    uint32_t out_blocks = 0;
    uint64_t out_bytes = 0;
    cudaEvent_t done_ev[2] = {};
    cudaEvent_t start_ev[2] = {};    // timing: device time of each tick
    Tick inflight[2];
    uint64_t tick_no = 0;
    // Ticks since the latest rebuild. A new batch cycles by plain launches;
    // it is captured into a CUDA graph once its membership has held for
    // kGraphAfter ticks, so sessions that come and go pay no capture.
    uint32_t same_ticks = 0;
    static constexpr uint32_t kGraphAfter = 8;
    // Statistics.
    std::vector<float> lat_ms;
    std::vector<float> tick_ms;          // device time of each tick (frames in to outputs out)
    float tick_max = 0;                  // the slowest tick: device ms, number, members, BM_TICK_* bits
    uint64_t tick_max_no = 0;
    uint32_t tick_max_members = 0, tick_max_what = 0;
    double tick_max_enq0 = 0, tick_max_enq1 = 0, tick_max_done = 0;   // its host-time window
    uint64_t ticks = 0, frames_cycled = 0, rebuilds = 0;
    uint64_t rebuild_drains = 0;         // rebuilds that waited for the queued ticks (staging blocks grew)
    double syn_cycles = 0, busy_s = 0, first_tick = 0, last_tick = 0;
    double rebuild_s = 0;                // host time in batch rebuilds
    double capture_s = 0;                // host time of the ticks that captured a batch's CUDA graph
    std::atomic<double> admit_s{0};      // builder-thread time in admissions
    double gpu_s = 0;                    // device time of the ticks (frames in to outputs out)
    // The builder thread and its queues (guarded by mu).
    std::thread builder;
    std::mutex mu;
    std::condition_variable cv;
    bool stop = false;
    std::deque<Session*> build_q;        // admitted sessions whose areas the builder builds
    // What the builder releases, in queue order: a retired batch (after the
    // ticks queued with it), a device buffer (likewise), a retired session's
    // area and output buffer. A session's batches are queued before its area.
    struct Teardown {
        bm_area area = nullptr;
        uint8_t* out = nullptr;
        bm_batch batch = nullptr;
        void* dev = nullptr;
    };
    std::deque<Teardown> free_q;
    // The builder's recent operations (guarded by mu): host-time span and
    // BM_BUILDER_* kind, to tell which ones overlapped a slow tick.
    struct BuilderOp {
        double t0, t1;
        uint32_t kind;
    };
    std::vector<BuilderOp> builder_ops;
    void log_op(double t0, uint32_t kind) {   // with mu held
        if (builder_ops.size() >= 8192) builder_ops.erase(builder_ops.begin(), builder_ops.begin() + 4096);
        builder_ops.push_back({t0, now_s(), kind});
    }

    Session* find(uint32_t id) {
        for (Session* s : sessions)
            if (s->id == id && !s->retired) return s;
        return nullptr;
    }
};

namespace {

void free_session(bm_server_s::Session* S) {
    if (S->area) bm_area_destroy(S->area);
    std::free(S->out);
    delete S;
}

// Builds S's area on the set-up context and its pinned output buffer (builder
// thread). The area is complete (grown, synchronised) when this returns.
int build_session(bm_server_s* V, bm_server_s::Session* S) {
    int rc = bm_area_create(V->setup, &S->desc, S->seed, &S->area);
    if (rc != BM_OK) return rc;
    // The gather-offset compile a new area's first cycle would run happens
    // here, on the set-up stream, not inside a tick.
    run_pending_verifies(S->area, V->setup->stream());
    const cudaError_t e = cudaStreamSynchronize(V->setup->stream());
    if (e != cudaSuccess) {
        bm_area_destroy(S->area);
        S->area = nullptr;
        return cuda_err(e, "session set-up");
    }
    // The latest output, copied out of the pinned gather block on the host:
    // plain memory (no page-locking, whose release would synchronize the
    // device beside the ticks).
    S->out = (uint8_t*)std::malloc(S->out_len ? S->out_len : 1);
    if (!S->out) {
        bm_area_destroy(S->area);
        S->area = nullptr;
        return set_err(BM_ERR_OOM, "pinned output buffer");
    }
    std::memset(S->out, 0, S->out_len ? S->out_len : 1);
    return BM_OK;
}

// The builder thread: tears down retired sessions' areas and builds admitted
// sessions' areas, in queue order, until the server stops.
void builder_loop(bm_server_s* V, int device) {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(V->mu);
    for (;;) {
        V->cv.wait(lk, [&] { return V->stop || !V->build_q.empty() || !V->free_q.empty(); });
        if (!V->free_q.empty()) {
            const bm_server_s::Teardown T = V->free_q.front();
            V->free_q.pop_front();
            lk.unlock();
            const double t0 = now_s();
            uint32_t kind = 0;
            if (T.batch) {
                bm_batch_destroy(T.batch);   // waits for the serving stream first
                kind |= BM_BUILDER_BATCH;
            }
            if (T.dev) {
                dev_free(T.dev, true, V->serve->stream());   // behind the ticks that read it
                kind |= BM_BUILDER_DEVICE_BUFFER;
            }
            if (T.area) {
                bm_area_destroy(T.area);
                kind |= BM_BUILDER_AREA_FREE;
            }
            if (T.out) {
                std::free(T.out);
                kind |= BM_BUILDER_OUTPUT_FREE;
            }
            lk.lock();
            V->log_op(t0, kind);
            continue;
        }
        if (!V->build_q.empty()) {
            bm_server_s::Session* S = V->build_q.front();
            V->build_q.pop_front();
            lk.unlock();
            const double t0 = now_s();
            S->build_rc = build_session(V, S);
            if (S->build_rc != BM_OK) S->build_msg = bm_last_error();
            V->admit_s.store(V->admit_s.load() + (now_s() - t0));
            S->build.store(S->build_rc == BM_OK ? bm_server_s::kBuilt : bm_server_s::kFailed,
                           std::memory_order_release);
            lk.lock();
            V->log_op(t0, BM_BUILDER_BUILD);
            continue;
        }
        if (V->stop) return;
    }
}

// Device bytes a session holds while resident (slab, gather offsets of every
// tuft, control block and slice table), from its resolved plan.
uint64_t footprint(const bm_area_plan& P) {
    uint64_t b = P.slab_bytes + 2 * P.n_syns_total + sizeof(AreaCtl) + BM_MAX_SLICES * sizeof(SliceRec);
    return (b + 0xFFFFF) & ~0xFFFFFull;   // the allocator's 1 MiB-ish granularity, rounded up
}

// Reserves S's bytes and hands it to the builder thread.
void admit(bm_server_s* V, bm_server_s::Session* S) {
    V->used += S->bytes;
    S->build.store(bm_server_s::kQueued);
    {
        std::lock_guard<std::mutex> g(V->mu);
        V->build_q.push_back(S);
    }
    V->cv.notify_one();
}

// A built session joins the ticks: its area's later work goes to the serving
// stream (same device).
void adopt(bm_server_s* V, bm_server_s::Session* S) {
    ctx_retain(V->serve);
    ctx_release(S->area->ctx);
    S->area->ctx = V->serve;
    S->resident = true;
    S->admitted = now_s();
}

void hand_to_builder(bm_server_s* V, const bm_server_s::Teardown& T) {
    {
        std::lock_guard<std::mutex> g(V->mu);
        V->free_q.push_back(T);
    }
    V->cv.notify_one();
}

// Releases S's budget and hands its area and output buffer to the builder
// thread for teardown.
void retire(bm_server_s* V, bm_server_s::Session* S) {
    if (S->build.load() != bm_server_s::kWaiting) V->used -= S->bytes;
    S->resident = false;
    S->retired = true;
    if (S->area || S->out) {
        bm_server_s::Teardown T;
        T.area = S->area;
        T.out = S->out;
        hand_to_builder(V, T);
    }
    S->area = nullptr;
    S->out = nullptr;
}

// The current batch leaves the ticks: the builder destroys it once the ticks
// queued with it are done, so the tick thread does not wait for them.
void retire_batch(bm_server_s* V) {
    if (V->batch) {
        bm_server_s::Teardown T;
        T.batch = V->batch;
        hand_to_builder(V, T);
    }
    V->batch = nullptr;
    V->members.clear();
}

// Grows a pair of pinned blocks and their device block, by half again what
// is asked for (the stream must be idle: callers complete the queued ticks
// before a growth).
int ensure_blocks(bm_ctx serve, uint8_t* (&h)[2], uint8_t*& d, uint64_t& cap, uint64_t bytes, const char* what) {
    if (bytes <= cap) return BM_OK;
    for (auto& p : h)
        if (p) cudaFreeHost(p);
    dev_free(d, true, serve->stream());
    h[0] = h[1] = nullptr;
    d = nullptr;
    cap = 0;
    uint64_t c = std::max<uint64_t>(bytes + bytes / 2, 1 << 20);
    if (cudaHostAlloc(&h[0], c, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc(&h[1], c, cudaHostAllocDefault) != cudaSuccess || dev_alloc(serve, &d, c) != cudaSuccess) {
        cudaGetLastError();
        return set_err(BM_ERR_OOM, "%s staging of %llu bytes", what, (unsigned long long)c);
    }
    cap = c;
    return BM_OK;
}

// Completes queued tick slot b: latencies, outputs, counters.
int complete(bm_server_s* V, uint32_t b) {
    bm_server_s::Tick& T = V->inflight[b];
    if (!T.live) return BM_OK;
    cudaError_t e = cudaEventSynchronize(V->done_ev[b]);
    if (e != cudaSuccess) return cuda_err(e, "tick");
    const double t1 = now_s();
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, V->start_ev[b], V->done_ev[b]) == cudaSuccess) {
        V->gpu_s += ms * 1e-3;
        V->tick_ms.push_back(ms);
        if (ms > V->tick_max) {
            V->tick_max = ms;
            V->tick_max_no = T.no;
            V->tick_max_members = (uint32_t)T.members.size();
            V->tick_max_what = T.what;
            V->tick_max_enq0 = T.enq0;
            V->tick_max_enq1 = T.enq1;
            V->tick_max_done = t1;
        }
    }
    cudaGetLastError();
    uint64_t o = 0;
    for (size_t k = 0; k < T.members.size(); k++) {
        auto* S = T.members[k];
        std::memcpy(S->out, V->h_out[T.buf] + o, S->out_len);
        o += S->out_len;
        const double ready = std::max(T.submitted[k], S->last_done);
        V->lat_ms.push_back((float)((t1 - ready) * 1e3));
        S->done++;
        S->inflight--;
        S->last_done = t1;
    }
    V->ticks++;
    V->frames_cycled += T.members.size();
    V->syn_cycles += T.syn;
    V->busy_s += t1 - T.started;
    V->last_tick = t1;
    T.live = false;
    T.members.clear();
    T.submitted.clear();
    return BM_OK;
}

int complete_all(bm_server_s* V) {
    // Ticks complete in queue order: the older slot first (the latest queued
    // tick, tick_no - 1, sits in slot (tick_no - 1) & 1).
    const uint32_t older = (uint32_t)(V->tick_no & 1);
    int rc = complete(V, older);
    if (rc == BM_OK) rc = complete(V, older ^ 1);
    return rc;
}

// Output gather of the current batch's members, packed in batch order. The
// previous gather table may still be read by a queued tick: the builder frees
// it after that.
int build_outjobs(bm_server_s* V) {
    if (V->d_outjobs) {
        bm_server_s::Teardown T;
        T.dev = V->d_outjobs;
        hand_to_builder(V, T);
    }
    V->d_outjobs = nullptr;
    std::vector<OutJob> jobs;
    uint64_t blocks = 0, o = 0;
    for (auto* S : V->members) {
        OutJob J;
        J.src = S->area->axns() + S->area->plan.outputs[0].axn_idz;
        J.dst_off = o;
        J.len = S->out_len;
        J.block0 = (uint32_t)blocks;
        blocks += (J.len + kGatherBlock * 4 - 1) / (kGatherBlock * 4);
        o += J.len;
        jobs.push_back(J);
    }
    V->out_blocks = (uint32_t)blocks;
    V->out_bytes = o;
    if (o > V->out_cap) {
        int rc = complete_all(V);
        if (rc != BM_OK) return rc;
        V->rebuild_drains++;
    }
    int rc = ensure_blocks(V->serve, V->h_out, V->d_out, V->out_cap, o, "output");
    if (rc != BM_OK) return rc;
    cudaError_t e = dev_alloc(V->serve, &V->d_outjobs, jobs.size() * sizeof(OutJob));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(V->d_outjobs, jobs.data(), jobs.size() * sizeof(OutJob), cudaMemcpyHostToDevice,
                            V->serve->stream());
    if (e != cudaSuccess) return cuda_err(e, "output gather jobs");
    return BM_OK;
}

}  // namespace

extern "C" {

int bm_server_create(bm_ctx ctx, uint64_t mem_budget, bm_server* out) {
    if (!ctx || !out) return set_err(BM_ERR_INVALID, "bm_server_create: null argument");
    *out = nullptr;
    DevGuard g(ctx->device);
    bm_server_s* V = new (std::nothrow) bm_server_s;
    if (!V) return set_err(BM_ERR_OOM, "host allocation failed");
    int rc = bm_ctx_create(ctx->device, 0, &V->setup);
    if (rc != BM_OK) { delete V; return rc; }
    V->ctx = ctx;
    ctx_retain(ctx);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = ctx->device;
    V->serve = new (std::nothrow) bm_ctx_s;
    cudaError_t pe = V->serve ? cudaMemPoolCreate(&V->pool, &props) : cudaErrorMemoryAllocation;
    if (pe == cudaSuccess) {
        // Memory freed to the pool stays there for the next sessions.
        uint64_t keep = ~0ull;
        pe = cudaMemPoolSetAttribute(V->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (pe != cudaSuccess) {
        cudaGetLastError();
        if (V->pool) cudaMemPoolDestroy(V->pool);
        delete V->serve;
        bm_ctx_destroy(V->setup);
        ctx_release(V->ctx);
        delete V;
        return cuda_err(pe, "server memory pool");
    }
    V->serve->device = ctx->device;
    V->serve->user = ctx->stream();
    V->serve->user_set = true;
    V->serve->pool = V->pool;
    V->setup->pool = V->pool;
    if (!mem_budget) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        mem_budget = (uint64_t)(fr * 0.9);
    }
    V->budget = mem_budget;
    if (cudaEventCreate(&V->done_ev[0]) != cudaSuccess || cudaEventCreate(&V->done_ev[1]) != cudaSuccess ||
        cudaEventCreate(&V->start_ev[0]) != cudaSuccess || cudaEventCreate(&V->start_ev[1]) != cudaSuccess) {
        cudaGetLastError();
        for (int b = 0; b < 2; b++) {
            if (V->done_ev[b]) cudaEventDestroy(V->done_ev[b]);
            if (V->start_ev[b]) cudaEventDestroy(V->start_ev[b]);
        }
        ctx_release(V->serve);
        bm_ctx_destroy(V->setup);
        cudaMemPoolDestroy(V->pool);
        ctx_release(V->ctx);
        delete V;
        return set_err(BM_ERR_CUDA, "cudaEventCreate");
    }
    V->builder = std::thread(builder_loop, V, ctx->device);
    *out = V;
    return BM_OK;
}

int bm_server_destroy(bm_server V) {
    if (!V) return BM_OK;
    DevGuard g(V->ctx->device);
    {
        std::lock_guard<std::mutex> lk(V->mu);
        V->stop = true;
    }
    V->cv.notify_one();
    if (V->builder.joinable()) V->builder.join();   // it finishes its queues first
    cudaStreamSynchronize(V->ctx->stream());
    if (V->batch) bm_batch_destroy(V->batch);
    for (auto* S : V->sessions) free_session(S);
    for (int b = 0; b < 2; b++) {
        if (V->h_frames[b]) cudaFreeHost(V->h_frames[b]);
        if (V->h_out[b]) cudaFreeHost(V->h_out[b]);
        if (V->done_ev[b]) cudaEventDestroy(V->done_ev[b]);
        if (V->start_ev[b]) cudaEventDestroy(V->start_ev[b]);
    }
    dev_free(V->d_frames, true, V->serve->stream());
    dev_free(V->d_out, true, V->serve->stream());
    dev_free(V->d_outjobs, true, V->serve->stream());
    cudaStreamSynchronize(V->serve->stream());
    ctx_release(V->serve);
    bm_ctx_destroy(V->setup);
    // The pool's memory is released once every allocation from it is freed.
    cudaMemPoolDestroy(V->pool);
    ctx_release(V->ctx);
    delete V;
    return BM_OK;
}

int bm_server_open(bm_server V, const bm_area_desc* desc, uint64_t seed, uint32_t* session) {
    if (!V || !desc || !session) return set_err(BM_ERR_INVALID, "bm_server_open: null argument");
    bm_area_plan P;
    int rc = bm_plan_resolve(desc, seed, &P);
    if (rc != BM_OK) return rc;
    if (P.n_inputs != 1 || P.n_outputs < 1)
        return set_err(BM_ERR_UNSUPPORTED, "bm_server_open: a session's area needs exactly one input and an output layer");
    auto* S = new (std::nothrow) bm_server_s::Session;
    if (!S) return set_err(BM_ERR_OOM, "host allocation failed");
    S->id = V->next_id++;
    S->desc = *desc;
    S->seed = seed;
    S->bytes = footprint(P);
    S->in_len = P.inputs[0].len;
    S->out_len = P.outputs[0].len;
    S->opened = now_s();
    if (S->bytes > V->budget) {
        delete S;
        return set_err(BM_ERR_OOM, "bm_server_open: the session needs %llu device bytes, above the whole budget",
                       (unsigned long long)P.slab_bytes);
    }
    V->sessions.push_back(S);
    *session = S->id;
    return BM_OK;
}

int bm_server_submit(bm_server V, uint32_t session, const uint8_t* frames, size_t frame_len, uint32_t n_frames) {
    if (!V || (!frames && n_frames)) return set_err(BM_ERR_INVALID, "bm_server_submit: null argument");
    auto* S = V->find(session);
    if (!S) return set_err(BM_ERR_INVALID, "bm_server_submit: no open session %u", session);
    if (S->closing) return set_err(BM_ERR_INVALID, "bm_server_submit: session %u is closing", session);
    if (frame_len != S->in_len) return set_err(BM_ERR_INVALID, "frame length %zu != %u", frame_len, S->in_len);
    const double t = now_s();
    if (n_frames) {
        Chunk c;
        c.bytes.assign(frames, frames + (size_t)n_frames * frame_len);
        c.n = n_frames;
        c.submitted = t;
        S->frames.len = (uint32_t)frame_len;
        S->frames.chunks.push_back(std::move(c));
    }
    return BM_OK;
}

int bm_server_close(bm_server V, uint32_t session) {
    if (!V) return set_err(BM_ERR_INVALID, "null server");
    auto* S = V->find(session);
    if (!S) return set_err(BM_ERR_INVALID, "bm_server_close: no open session %u", session);
    S->closing = true;
    return BM_OK;
}

int bm_server_cancel(bm_server V, uint32_t session) {
    if (!V) return set_err(BM_ERR_INVALID, "null server");
    auto* S = V->find(session);
    if (!S) return set_err(BM_ERR_INVALID, "bm_server_cancel: no open session %u", session);
    S->closing = true;
    S->frames.chunks.clear();   // frames already in a queued tick still complete
    return BM_OK;
}

int bm_server_tick(bm_server V, uint32_t* n_cycled) {
    if (!V) return set_err(BM_ERR_INVALID, "null server");
    DevGuard g(V->ctx->device);
    cudaStream_t s = V->ctx->stream();
    V->serve->user = s;   // the serving stream, should the caller have changed it
    const double t0 = now_s();
    if (!V->first_tick) V->first_tick = t0;

    // 0. A session whose area ended a cycle with device error bits (a bounded
    //    wait in a kernel gave up) is dropped with its queued frames; the
    //    tick reports it once, after the queued ticks complete, and the next
    //    tick runs the other sessions without it.
    {
        uint32_t n_failed = 0, first = 0;
        unsigned int bits = 0;
        for (auto* S : V->sessions) {
            if (!S->resident || S->failed || !S->area) continue;
            const unsigned int e = S->area->seen_errors();
            if (!e) continue;
            S->failed = true;
            S->closing = true;
            S->frames.chunks.clear();
            V->failed_ids.push_back(S->id);
            if (!n_failed++) { first = S->id; bits = e; }
        }
        if (n_failed) {
            const int rc = complete_all(V);
            if (rc != BM_OK) return rc;
            return set_err(BM_ERR_TIMEOUT,
                           "bm_server_tick: session %u ended a cycle with device error bits 0x%x and was dropped "
                           "(%u session(s) this tick)", first, bits, n_failed);
        }
    }

    // 1. Retire drained, closed sessions (no frame left, none in flight, not
    //    with the builder). A batch that holds one is dropped first.
    for (auto* S : V->sessions) {
        if (!S->closing || !S->frames.empty() || S->inflight) continue;
        if (S->build.load(std::memory_order_acquire) == bm_server_s::kQueued) continue;
        if (std::find(V->members.begin(), V->members.end(), S) != V->members.end()) retire_batch(V);
        retire(V, S);
    }
    std::vector<bm_server_s::Session*> live;
    for (auto* S : V->sessions)
        if (!S->retired) live.push_back(S);
        else free_session(S);
    V->sessions.swap(live);

    // 2. Adopt the sessions the builder finished, then queue tick N: resident
    //    sessions with a pending frame.
    for (auto* S : V->sessions) {
        if (S->resident || S->retired) continue;
        const int b = S->build.load(std::memory_order_acquire);
        if (b == bm_server_s::kBuilt) adopt(V, S);
        else if (b == bm_server_s::kFailed) {
            // Reported once; the session waits for admission again.
            V->used -= S->bytes;
            S->build.store(bm_server_s::kWaiting);
            return set_err(S->build_rc, "bm_server_tick: building session %u failed: %s", S->id,
                           S->build_msg.c_str());
        }
    }
    // A session whose area shows device error bits is left out (the next
    // tick drops it); the batch then runs without checking them again, so a
    // bit that appears after this check cannot strand the tick's frames.
    std::vector<bm_server_s::Session*> m;
    for (auto* S : V->sessions)
        if (S->resident && !S->frames.empty() && !S->area->seen_errors()) m.push_back(S);
    if (n_cycled) *n_cycled = (uint32_t)m.size();
    const uint32_t slot = (uint32_t)(V->tick_no & 1);
    uint32_t what = V->tick_no == 0 ? BM_TICK_FIRST : 0u;
    if (!m.empty()) {
        if (m != V->members || !V->batch) {
            what |= BM_TICK_REBUILD;
            // A new batch for the new membership; the previous tick stays
            // queued (its batch and gather table are released behind it),
            // unless a staging block must grow.
            const double r0 = now_s();
            retire_batch(V);
            std::vector<bm_area> areas;
            for (auto* S : m) areas.push_back(S->area);
            int rc = bm_batch_create(V->serve, areas.data(), (uint32_t)areas.size(), &V->batch);
            if (rc == BM_OK) rc = bm_batch_set_graph(V->batch, 0);
            if (rc != BM_OK) return rc;
            V->same_ticks = 0;
            V->members = m;
            V->rebuilds++;
            uint64_t fb = 0;
            bm_batch_frame_bytes(V->batch, &fb);
            if (fb > V->frames_cap) {
                rc = complete_all(V);
                if (rc != BM_OK) return rc;
                V->rebuild_drains++;
                what |= BM_TICK_DRAIN;
            }
            rc = ensure_blocks(V->serve, V->h_frames, V->d_frames, V->frames_cap, fb, "frame");
            if (rc == BM_OK) rc = build_outjobs(V);
            if (rc != BM_OK) return rc;
            V->rebuild_s += now_s() - r0;
        }
        // Slot `slot` was completed at least one call ago, so its pinned
        // blocks are free.
        bm_server_s::Tick& T = V->inflight[slot];
        T.live = true;
        T.buf = slot;
        T.started = t0;
        T.syn = 0;
        T.members = m;
        T.no = V->tick_no;
        uint64_t o = 0;
        for (auto* S : m) {
            std::memcpy(V->h_frames[slot] + o, S->frames.front(), S->in_len);
            o += S->in_len;
            T.submitted.push_back(S->frames.front_submitted());
            T.syn += (double)S->area->plan.n_syns_total;
            S->frames.pop();
            S->inflight++;
        }
        T.enq0 = now_s();
        cudaError_t e = cudaEventRecord(V->start_ev[slot], s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(V->d_frames, V->h_frames[slot], o, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_err(e, "frame block copy");
        const bool capture = ++V->same_ticks == bm_server_s::kGraphAfter;
        const double c0 = capture ? now_s() : 0.0;
        if (capture) {
            int rc = bm_batch_set_graph(V->batch, 1);
            if (rc != BM_OK) return rc;
        }
        int rc = batch_cycle_frames_unchecked(V->batch, V->d_frames);
        if (rc != BM_OK) return rc;
        if (capture) {
            V->capture_s += now_s() - c0;
            what |= BM_TICK_CAPTURE;
        }
        T.what = what;
        if (V->out_blocks) k_gather_outputs<<<V->out_blocks, kGatherBlock, 0, s>>>(V->d_outjobs, (uint32_t)m.size(), V->d_out);
        e = cudaMemcpyAsync(V->h_out[slot], V->d_out, V->out_bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaEventRecord(V->done_ev[slot], s);
        if (e != cudaSuccess) return cuda_err(e, "tick");
        T.enq1 = now_s();
        V->tick_no++;
    }

    // 3. Admit waiting sessions in FIFO order as the budget allows (none
    //    overtakes an earlier one that does not fit). The builder thread
    //    builds their areas; they join the first tick after it is done.
    for (auto* S : V->sessions) {
        if (S->resident || S->build.load() != bm_server_s::kWaiting || S->retired) continue;
        if (V->used + S->bytes > V->budget) break;
        admit(V, S);
    }

    // 4. Complete the previous tick (with nothing queued now: every tick).
    if (!m.empty()) return complete(V, slot ^ 1);
    return complete_all(V);
}

int bm_server_drain(bm_server V) {
    if (!V) return set_err(BM_ERR_INVALID, "null server");
    DevGuard g(V->ctx->device);
    return complete_all(V);
}

int bm_server_read_output(bm_server V, uint32_t session, uint8_t* dst, size_t len, uint64_t* frames_done) {
    if (!V || !dst) return set_err(BM_ERR_INVALID, "null argument");
    auto* S = V->find(session);
    const bool failed = S ? S->failed
                          : std::find(V->failed_ids.begin(), V->failed_ids.end(), session) != V->failed_ids.end();
    if (failed)
        return set_err(BM_ERR_TIMEOUT, "bm_server_read_output: session %u was dropped after a device error", session);
    if (!S) return set_err(BM_ERR_INVALID, "bm_server_read_output: no open session %u", session);
    if (len != S->out_len) return set_err(BM_ERR_INVALID, "length %zu != %u", len, S->out_len);
    if (S->out) std::memcpy(dst, S->out, len);
    else std::memset(dst, 0, len);
    if (frames_done) *frames_done = S->done;
    return BM_OK;
}

int bm_server_session_area(bm_server V, uint32_t session, bm_area* out) {
    if (!V || !out) return set_err(BM_ERR_INVALID, "null argument");
    auto* S = V->find(session);
    if (!S) return set_err(BM_ERR_INVALID, "no open session %u", session);
    *out = S->area;
    return BM_OK;
}

int bm_server_get_stats(bm_server V, bm_server_stats* st) {
    if (!V || !st) return set_err(BM_ERR_INVALID, "null argument");
    std::memset(st, 0, sizeof *st);
    st->ticks = V->ticks;
    st->frames = V->frames_cycled;
    st->batch_rebuilds = V->rebuilds;
    st->syn_cycles = V->syn_cycles;
    st->busy_s = V->busy_s;
    st->span_s = V->last_tick > V->first_tick ? V->last_tick - V->first_tick : 0;
    st->rebuild_s = V->rebuild_s;
    st->rebuild_drains = V->rebuild_drains;
    st->capture_s = V->capture_s;
    st->gpu_s = V->gpu_s;
    st->admit_s = V->admit_s.load();
    st->used_bytes = V->used;
    st->budget_bytes = V->budget;
    for (auto* S : V->sessions) {
        if (S->resident) st->resident++;
        else st->waiting++;
    }
    st->failed = (uint32_t)V->failed_ids.size();
    if (!V->lat_ms.empty()) {
        std::vector<float> v = V->lat_ms;
        auto q = [&](double f) {
            size_t k = (size_t)(f * (v.size() - 1) + 0.5);
            std::nth_element(v.begin(), v.begin() + k, v.end());
            return (double)v[k];
        };
        st->p50_ms = q(0.50);
        st->p99_ms = q(0.99);
        if (!V->tick_ms.empty()) {
            std::vector<float> t = V->tick_ms;
            const size_t k = (size_t)(0.99 * (t.size() - 1) + 0.5);
            std::nth_element(t.begin(), t.begin() + k, t.end());
            st->tick_p99_ms = t[k];
            st->tick_max_ms = V->tick_max;
            st->tick_max_no = V->tick_max_no;
            st->tick_max_members = V->tick_max_members;
            st->tick_max_what = V->tick_max_what;
            st->tick_max_queue_ms = (V->tick_max_enq1 - V->tick_max_enq0) * 1e3;
            std::lock_guard<std::mutex> g(V->mu);
            for (const auto& op : V->builder_ops) {
                if (op.t1 < V->tick_max_enq0 || op.t0 > V->tick_max_done) continue;
                st->tick_max_builder |= op.kind;
                st->tick_max_builder_ms = std::max(st->tick_max_builder_ms, (op.t1 - op.t0) * 1e3);
            }
        }
        double sum = 0;
        for (float x : V->lat_ms) sum += x;
        st->mean_ms = sum / V->lat_ms.size();
    }
    return BM_OK;
}

int bm_server_reset_stats(bm_server V) {
    if (!V) return set_err(BM_ERR_INVALID, "null server");
    V->lat_ms.clear();
    V->tick_ms.clear();
    V->tick_max = 0;
    V->tick_max_no = 0;
    V->tick_max_members = V->tick_max_what = 0;
    V->tick_max_enq0 = V->tick_max_enq1 = V->tick_max_done = 0;
    V->ticks = V->frames_cycled = V->rebuilds = V->rebuild_drains = 0;
    V->syn_cycles = V->busy_s = V->first_tick = V->last_tick = V->rebuild_s = V->gpu_s = V->capture_s = 0;
    V->admit_s.store(0);
    return BM_OK;
}

}  // extern "C"
