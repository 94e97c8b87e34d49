// bm_sampler.cu -- samplers: per-cycle readback of one buffer of an area.
//
// CorticalArea::sampler (src/cortex/cortical_area.rs:1017-1284, with
// SamplerBufferKind::Single, the only kind the reference implements) gives a
// receiver a one-frame channel over a whole layer buffer, or over the axons
// of one layer or of the area. After every cycle the area sends the buffer
// (CorticalArea::cycle_samplers, :809-880) through that channel, which
// behaves as the reference's tract channel (src/subcortex/tract_channel.rs:
// 400-488):
//   * no unread frame: the new frame is sent;
//   * an unread frame and no backpressure: the new frame is skipped (the
//     receiver later gets the older, unread one);
//   * an unread frame and backpressure: the cycling thread waits until the
//     receiver takes it, then sends.
// recv(wait_for_frame) takes the unread frame, or waits for the next send, or
// returns none.
//
// Here a send is a device copy of the range, enqueued on the cycling stream
// after the cycle's kernels, then a device-to-host copy of it into the
// sampler's pinned frame buffer on a stream of its own (so the next cycle
// does not wait for it), with an event the receiver waits on. The channel
// state is a mutex
// and a condition variable shared by the cycling and the receiving thread.
// A wait may be bounded (bm_sampler_set_timeout); the reference waits forever,
// which is also the default.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <new>

#include "bm_area.h"

using namespace bm;

struct bm_sampler_s {
    bm_area area = nullptr;
    uint64_t off = 0, len = 0;   // sampled range of the area's state slab
    uint8_t* host = nullptr;     // pinned frame buffer
    uint8_t* dev = nullptr;      // device copy of the range (ranges up to kStageMax)
    cudaEvent_t staged = nullptr;  // the device copy is taken
    cudaEvent_t done = nullptr;  // the frame's copy has landed
    std::mutex mu;
    std::condition_variable cv;
    bool ready = false;          // a frame waits for the receiver
    bool backpressure = false;
    uint64_t frame_cycle = 0;    // cycle whose end state the frame holds
    uint64_t sent = 0, skipped = 0;
    uint32_t timeout_ms = 0;     // bounded waits (0: wait forever)
};

namespace {

// Ranges up to this size are first copied on the device, on the cycling
// stream, and downloaded on the area's `down` stream beside the next cycle;
// larger ones are downloaded on the cycling stream directly.
constexpr uint64_t kStageMax = 64ull << 20;

template <class Pred>
bool wait_for(bm_sampler_s* S, std::unique_lock<std::mutex>& lk, Pred pred) {
    if (!S->timeout_ms) {
        S->cv.wait(lk, pred);
        return true;
    }
    return S->cv.wait_for(lk, std::chrono::milliseconds(S->timeout_ms), pred);
}

void destroy_sampler(bm_sampler_s* S) {
    if (S->done) {
        cudaEventSynchronize(S->done);
        cudaEventDestroy(S->done);
    }
    if (S->staged) cudaEventDestroy(S->staged);
    if (S->dev) cudaFree(S->dev);
    if (S->host) cudaFreeHost(S->host);
    delete S;
}

}  // namespace

void bm::sampler_range(const bm_sampler_s* S, uint64_t* off, uint64_t* len) {
    *off = S->off;
    *len = S->len;
}

int bm::sample_after_cycle(bm_area_s* A, cudaStream_t s) {
    for (bm_sampler_s* S : A->samplers) {
        std::unique_lock<std::mutex> lk(S->mu);
        if (S->ready) {
            if (!S->backpressure) {
                S->skipped++;
                continue;
            }
            if (!wait_for(S, lk, [&] { return !S->ready || !S->backpressure; }))
                return set_err(BM_ERR_TIMEOUT, "sampler: no receiver took the unread frame within %u ms",
                               S->timeout_ms);
            if (S->ready) {   // backpressure switched off while waiting
                S->skipped++;
                continue;
            }
        }
        cudaError_t e;
        if (S->dev) {
            // The previous download has left S->dev (long since: its frame
            // was taken or this one would be skipped).
            e = cudaStreamWaitEvent(s, S->done, 0);
            if (e == cudaSuccess) e = cudaMemcpyAsync(S->dev, A->slab + S->off, S->len, cudaMemcpyDeviceToDevice, s);
            if (e == cudaSuccess) e = cudaEventRecord(S->staged, s);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(A->down, S->staged, 0);
            if (e == cudaSuccess) e = cudaMemcpyAsync(S->host, S->dev, S->len, cudaMemcpyDeviceToHost, A->down);
            if (e == cudaSuccess) e = cudaEventRecord(S->done, A->down);
        } else {
            e = cudaMemcpyAsync(S->host, A->slab + S->off, S->len, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaEventRecord(S->done, s);
        }
        if (e != cudaSuccess) return cuda_err(e, "sampler copy");
        S->ready = true;
        S->frame_cycle = A->host_cycle - 1;
        S->sent++;
        S->cv.notify_all();
    }
    return BM_OK;
}

void bm::free_samplers(bm_area_s* A) {
    for (bm_sampler_s* S : A->samplers) destroy_sampler(S);
    A->samplers.clear();
}

extern "C" {

int bm_sampler_create(bm_area area, uint32_t kind, uint32_t layer, int backpressure, bm_sampler* out) {
    if (!area || !out) return set_err(BM_ERR_INVALID, "bm_sampler_create: null argument");
    *out = nullptr;
    const bm_area_plan& P = area->plan;
    uint64_t off = 0, len = 0;
    if (kind == BM_BUF_AXON_STATES) {
        // Axons of one layer (its slices, consecutive in the axon space) or
        // of the whole area (SamplerKind::Axons, :1031-1050).
        if (layer == BM_ALL_LAYERS) {
            off = P.axon_off;
            len = P.n_axons;
        } else {
            if (layer >= P.n_layers) return set_err(BM_ERR_INVALID, "sampler: layer %u out of range", layer);
            const bm_layer_plan& L = P.layers[layer];
            if (L.depth == 0 || L.base_axn_slc + L.depth > P.n_slices)
                return set_err(BM_ERR_INVALID, "sampler: layer %u has no axon slices", layer);
            const uint32_t k0 = L.base_axn_slc, k1 = L.base_axn_slc + L.depth - 1;
            const uint64_t a0 = P.slc_axn_idz[k0];
            const uint64_t a1 = (uint64_t)P.slc_axn_idz[k1] + (uint64_t)P.slc_v_size[k1] * P.slc_u_size[k1];
            uint64_t sum = 0;
            for (uint32_t k = k0; k <= k1; k++) sum += (uint64_t)P.slc_v_size[k] * P.slc_u_size[k];
            if (a1 - a0 != sum) return set_err(BM_ERR_INVALID, "sampler: layer %u slices are not contiguous", layer);
            off = P.axon_off + a0;
            len = sum;
        }
    } else {
        // A whole buffer of one data layer, every tuft (SomaStates ..
        // SynFlagSets, :1053-1284).
        if (kind >= BM_BUF_COUNT) return set_err(BM_ERR_INVALID, "sampler: unknown buffer kind %u", kind);
        if (layer >= P.n_layers) return set_err(BM_ERR_INVALID, "sampler: layer %u out of range", layer);
        const bm_layer_plan& L = P.layers[layer];
        if (L.buf_off[kind] == UINT64_MAX)
            return set_err(BM_ERR_INVALID, "sampler: layer %u has no buffer of kind %u", layer, kind);
        off = L.buf_off[kind];
        len = L.buf_len[kind];
    }
    if (len == 0) return set_err(BM_ERR_INVALID, "sampler: empty range");
    DevGuard g(area->ctx->device);
    bm_sampler_s* S = new (std::nothrow) bm_sampler_s;
    if (!S) return set_err(BM_ERR_OOM, "host allocation failed");
    S->area = area;
    S->off = off;
    S->len = len;
    S->backpressure = backpressure != 0;
    cudaError_t e = cudaHostAlloc((void**)&S->host, len, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->done, cudaEventDisableTiming);
    if (e == cudaSuccess && len <= kStageMax) {
        e = cudaMalloc(&S->dev, len);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->staged, cudaEventDisableTiming);
        if (e == cudaSuccess && !area->down) e = cudaStreamCreateWithFlags(&area->down, cudaStreamNonBlocking);
    }
    if (e != cudaSuccess) {
        destroy_sampler(S);
        return cuda_err(e, "sampler set-up");
    }
    area->samplers.push_back(S);
    *out = S;
    return BM_OK;
}

int bm_sampler_destroy(bm_sampler sampler) {
    if (!sampler) return BM_OK;
    bm_area A = sampler->area;
    DevGuard g(A->ctx->device);
    for (size_t k = 0; k < A->samplers.size(); k++)
        if (A->samplers[k] == sampler) {
            A->samplers.erase(A->samplers.begin() + (long)k);
            break;
        }
    destroy_sampler(sampler);
    return BM_OK;
}

int bm_sampler_len(bm_sampler sampler, uint64_t* len) {
    if (!sampler || !len) return set_err(BM_ERR_INVALID, "null argument");
    *len = sampler->len;
    return BM_OK;
}

int bm_sampler_set_backpressure(bm_sampler sampler, int on, int* prior) {
    if (!sampler) return set_err(BM_ERR_INVALID, "null sampler");
    std::lock_guard<std::mutex> lk(sampler->mu);
    if (prior) *prior = sampler->backpressure ? 1 : 0;
    sampler->backpressure = on != 0;
    sampler->cv.notify_all();
    return BM_OK;
}

int bm_sampler_set_timeout(bm_sampler sampler, uint32_t ms) {
    if (!sampler) return set_err(BM_ERR_INVALID, "null sampler");
    std::lock_guard<std::mutex> lk(sampler->mu);
    sampler->timeout_ms = ms;
    return BM_OK;
}

int bm_sampler_recv(bm_sampler sampler, int wait_for_frame, void* dst, uint64_t len, uint64_t* cycle, int* got) {
    if (!sampler || !dst || !got) return set_err(BM_ERR_INVALID, "null argument");
    if (len != sampler->len) return set_err(BM_ERR_INVALID, "sampler: frame is %llu bytes, not %llu",
                                            (unsigned long long)sampler->len, (unsigned long long)len);
    *got = 0;
    bm_sampler_s* S = sampler;
    std::unique_lock<std::mutex> lk(S->mu);
    if (!S->ready) {
        if (!wait_for_frame) return BM_OK;
        if (!wait_for(S, lk, [&] { return S->ready; }))
            return set_err(BM_ERR_TIMEOUT, "sampler: no frame within %u ms", S->timeout_ms);
    }
    // The frame stays unread (ready) while the receiver waits for its copy
    // and takes it, so a sender meanwhile skips or waits as for any unread
    // frame; the lock is not held across the device wait, so a sender without
    // backpressure never blocks on it.
    const uint64_t frame_cycle = S->frame_cycle;
    lk.unlock();
    DevGuard g(S->area->ctx->device);
    cudaError_t e = cudaEventSynchronize(S->done);
    if (e != cudaSuccess) return cuda_err(e, "sampler frame");
    std::memcpy(dst, S->host, S->len);
    if (cycle) *cycle = frame_cycle;
    *got = 1;
    lk.lock();
    S->ready = false;
    S->cv.notify_all();
    return BM_OK;
}

int bm_sampler_stats(bm_sampler sampler, uint64_t* sent, uint64_t* skipped) {
    if (!sampler) return set_err(BM_ERR_INVALID, "null sampler");
    std::lock_guard<std::mutex> lk(sampler->mu);
    if (sent) *sent = sampler->sent;
    if (skipped) *skipped = sampler->skipped;
    return BM_OK;
}

}  // extern "C"
