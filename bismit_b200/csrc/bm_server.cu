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
// one pinned block and copied in with one transfer; each session's output
// axons come back into its own pinned buffer. While a tick runs on the GPU the
// host admits waiting sessions: their areas are built and grown on a second
// stream, so set-up overlaps the running cycles.
//
// Latency of a frame = completion of the tick that cycled it minus the moment
// it became ready (its submission, or the completion of the session's
// previous frame if that came later): admission waits show up in it.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <new>
#include <vector>

#include "bm_area.h"

using namespace bm;

namespace {

using Clock = std::chrono::steady_clock;

double now_s() { return std::chrono::duration<double>(Clock::now().time_since_epoch()).count(); }

struct Frame {
    std::vector<uint8_t> bytes;
    double submitted;
};

}  // namespace

struct bm_server_s {
    struct Session {
        uint32_t id = 0;
        bm_area_desc desc;
        uint64_t seed = 0;
        uint64_t bytes = 0;          // device bytes while resident
        bm_area area = nullptr;
        std::deque<Frame> frames;
        uint8_t* out = nullptr;      // pinned: output 0 after the latest cycled frame
        uint32_t out_len = 0, in_len = 0;
        uint64_t done = 0;           // frames cycled
        double last_done = 0;        // completion time of the latest cycled frame
        double opened = 0, admitted = 0;
        bool closing = false, resident = false, retired = false;
    };
    bm_ctx ctx = nullptr;            // the serving stream
    bm_ctx setup = nullptr;          // area construction, overlapping the ticks
    uint64_t budget = 0, used = 0;
    uint32_t next_id = 1;
    std::vector<Session*> sessions;  // every open session, in open order
    bm_batch batch = nullptr;
    std::vector<Session*> members;   // the batch's sessions, in batch order
    uint8_t* h_frames = nullptr;     // pinned frame block
    uint8_t* d_frames = nullptr;
    uint64_t frames_cap = 0;
    cudaEvent_t done_ev = nullptr;
    // Statistics.
    std::vector<float> lat_ms;
    uint64_t ticks = 0, frames_cycled = 0, rebuilds = 0;
    double syn_cycles = 0, busy_s = 0, first_tick = 0, last_tick = 0;

    Session* find(uint32_t id) {
        for (Session* s : sessions)
            if (s->id == id && !s->retired) return s;
        return nullptr;
    }
};

namespace {

void free_session(bm_server_s::Session* S) {
    if (S->area) bm_area_destroy(S->area);
    if (S->out) cudaFreeHost(S->out);
    delete S;
}

// Device bytes a session holds while resident (slab, gather offsets of every
// tuft, control block and slice table), from its resolved plan.
uint64_t footprint(const bm_area_plan& P) {
    uint64_t b = P.slab_bytes + 2 * P.n_syns_total + sizeof(AreaCtl) + BM_MAX_SLICES * sizeof(SliceRec);
    return (b + 0xFFFFF) & ~0xFFFFFull;   // the allocator's 1 MiB-ish granularity, rounded up
}

// Builds the area of S on the set-up context and moves it to the serving one.
int admit(bm_server_s* V, bm_server_s::Session* S) {
    int rc = bm_area_create(V->setup, &S->desc, S->seed, &S->area);
    if (rc != BM_OK) return rc;
    S->area->ctx = V->ctx;   // same device; later work goes to the serving stream
    if (cudaHostAlloc(&S->out, S->out_len ? S->out_len : 1, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        bm_area_destroy(S->area);
        S->area = nullptr;
        return set_err(BM_ERR_OOM, "pinned output buffer");
    }
    std::memset(S->out, 0, S->out_len ? S->out_len : 1);
    S->resident = true;
    S->admitted = now_s();
    V->used += S->bytes;
    return BM_OK;
}

void retire(bm_server_s* V, bm_server_s::Session* S) {
    if (S->resident) V->used -= S->bytes;
    S->resident = false;
    S->retired = true;
    if (S->area) bm_area_destroy(S->area);
    S->area = nullptr;
}

int ensure_frames(bm_server_s* V, uint64_t bytes) {
    if (bytes <= V->frames_cap) return BM_OK;
    if (V->h_frames) cudaFreeHost(V->h_frames);
    if (V->d_frames) cudaFree(V->d_frames);
    V->h_frames = nullptr;
    V->d_frames = nullptr;
    V->frames_cap = 0;
    uint64_t cap = std::max<uint64_t>(bytes, 1 << 20);
    if (cudaHostAlloc(&V->h_frames, cap, cudaHostAllocDefault) != cudaSuccess || cudaMalloc(&V->d_frames, cap) != cudaSuccess) {
        cudaGetLastError();
        return set_err(BM_ERR_OOM, "frame staging of %llu bytes", (unsigned long long)cap);
    }
    V->frames_cap = cap;
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
    V->ctx = ctx;
    int rc = bm_ctx_create(ctx->device, 0, &V->setup);
    if (rc != BM_OK) { delete V; return rc; }
    if (!mem_budget) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        mem_budget = (uint64_t)(fr * 0.9);
    }
    V->budget = mem_budget;
    if (cudaEventCreateWithFlags(&V->done_ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        bm_ctx_destroy(V->setup);
        delete V;
        return set_err(BM_ERR_CUDA, "cudaEventCreate");
    }
    *out = V;
    return BM_OK;
}

int bm_server_destroy(bm_server V) {
    if (!V) return BM_OK;
    DevGuard g(V->ctx->device);
    cudaStreamSynchronize(V->ctx->stream());
    if (V->batch) bm_batch_destroy(V->batch);
    for (auto* S : V->sessions) free_session(S);
    if (V->h_frames) cudaFreeHost(V->h_frames);
    if (V->d_frames) cudaFree(V->d_frames);
    if (V->done_ev) cudaEventDestroy(V->done_ev);
    bm_ctx_destroy(V->setup);
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
    for (uint32_t k = 0; k < n_frames; k++) S->frames.push_back({std::vector<uint8_t>(frames + k * frame_len, frames + (k + 1) * frame_len), t});
    return BM_OK;
}

int bm_server_close(bm_server V, uint32_t session) {
    if (!V) return set_err(BM_ERR_INVALID, "null server");
    auto* S = V->find(session);
    if (!S) return set_err(BM_ERR_INVALID, "bm_server_close: no open session %u", session);
    S->closing = true;
    return BM_OK;
}

int bm_server_tick(bm_server V, uint32_t* n_cycled) {
    if (!V) return set_err(BM_ERR_INVALID, "null server");
    DevGuard g(V->ctx->device);
    cudaStream_t s = V->ctx->stream();
    const double t0 = now_s();
    if (!V->first_tick) V->first_tick = t0;

    // 1. Retire drained, closed sessions (their last tick has completed). A
    //    batch that holds one is dropped first.
    for (auto* S : V->sessions) {
        if (!S->closing || !S->frames.empty()) continue;
        if (std::find(V->members.begin(), V->members.end(), S) != V->members.end()) {
            if (V->batch) bm_batch_destroy(V->batch);
            V->batch = nullptr;
            V->members.clear();
        }
        retire(V, S);
    }
    std::vector<bm_server_s::Session*> live;
    for (auto* S : V->sessions)
        if (!S->retired) live.push_back(S);
        else free_session(S);
    V->sessions.swap(live);

    // 2. This tick's sessions: resident with a pending frame. Frames in, one
    //    batched cycle, outputs out, all queued on the serving stream.
    std::vector<bm_server_s::Session*> m;
    for (auto* S : V->sessions)
        if (S->resident && !S->frames.empty()) m.push_back(S);
    if (n_cycled) *n_cycled = (uint32_t)m.size();
    double syn = 0;
    if (!m.empty()) {
        if (m != V->members || !V->batch) {
            if (V->batch) bm_batch_destroy(V->batch);
            V->batch = nullptr;
            V->members.clear();
            std::vector<bm_area> areas;
            for (auto* S : m) areas.push_back(S->area);
            int rc = bm_batch_create(V->ctx, areas.data(), (uint32_t)areas.size(), &V->batch);
            if (rc != BM_OK) return rc;
            V->members = m;
            V->rebuilds++;
        }
        uint64_t fb = 0;
        bm_batch_frame_bytes(V->batch, &fb);
        int rc = ensure_frames(V, fb);
        if (rc != BM_OK) return rc;
        uint64_t o = 0;
        for (auto* S : m) {
            std::memcpy(V->h_frames + o, S->frames.front().bytes.data(), S->in_len);
            o += S->in_len;
            syn += (double)S->area->plan.n_syns_total;
        }
        cudaError_t e = cudaMemcpyAsync(V->d_frames, V->h_frames, fb, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_err(e, "frame block copy");
        rc = bm_batch_cycle_frames_device(V->batch, V->d_frames, 1);
        if (rc != BM_OK) return rc;
        for (auto* S : m) {
            const bm_io_plan& out = S->area->plan.outputs[0];
            e = cudaMemcpyAsync(S->out, S->area->axns() + out.axn_idz, out.len, cudaMemcpyDeviceToHost, s);
            if (e != cudaSuccess) return cuda_err(e, "output copy");
        }
        e = cudaEventRecord(V->done_ev, s);
        if (e != cudaSuccess) return cuda_err(e, "cudaEventRecord");
    }

    // 3. While that runs: admit waiting sessions in FIFO order as the budget
    //    allows (none overtakes an earlier one that does not fit). Their areas
    //    are built and grown on the set-up stream; they join the next tick.
    for (auto* S : V->sessions) {
        if (S->resident) continue;
        if (V->used + S->bytes > V->budget) break;
        int rc = admit(V, S);
        if (rc != BM_OK) return rc;
    }
    if (m.empty()) return BM_OK;

    // 4. Completion.
    cudaError_t e = cudaEventSynchronize(V->done_ev);
    if (e != cudaSuccess) return cuda_err(e, "tick");
    const double t1 = now_s();
    for (auto* S : m) {
        const Frame& f = S->frames.front();
        const double ready = std::max(f.submitted, S->last_done);
        V->lat_ms.push_back((float)((t1 - ready) * 1e3));
        S->frames.pop_front();
        S->done++;
        S->last_done = t1;
    }
    V->ticks++;
    V->frames_cycled += m.size();
    V->syn_cycles += syn;
    V->busy_s += t1 - t0;
    V->last_tick = t1;
    return BM_OK;
}

int bm_server_read_output(bm_server V, uint32_t session, uint8_t* dst, size_t len, uint64_t* frames_done) {
    if (!V || !dst) return set_err(BM_ERR_INVALID, "null argument");
    auto* S = V->find(session);
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
    st->used_bytes = V->used;
    st->budget_bytes = V->budget;
    for (auto* S : V->sessions) {
        if (S->resident) st->resident++;
        else st->waiting++;
    }
    if (!V->lat_ms.empty()) {
        std::vector<float> v = V->lat_ms;
        auto q = [&](double f) {
            size_t k = (size_t)(f * (v.size() - 1) + 0.5);
            std::nth_element(v.begin(), v.begin() + k, v.end());
            return (double)v[k];
        };
        st->p50_ms = q(0.50);
        st->p99_ms = q(0.99);
        double sum = 0;
        for (float x : V->lat_ms) sum += x;
        st->mean_ms = sum / V->lat_ms.size();
    }
    return BM_OK;
}

int bm_server_reset_stats(bm_server V) {
    if (!V) return set_err(BM_ERR_INVALID, "null server");
    V->lat_ms.clear();
    V->ticks = V->frames_cycled = V->rebuilds = 0;
    V->syn_cycles = V->busy_s = V->first_tick = V->last_tick = 0;
    return BM_OK;
}

}  // extern "C"
