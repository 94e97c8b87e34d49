// bm_static.cu -- bm_tuft_cycle_static: one fused tuft cycle (synapse flags,
// synapse cycle, dendrite cycle, and the tuft cycle for pyramidal layers) on a
// state slab the caller owns, with no device allocation at any point.
//
// Who needs it: callers that are not allowed to allocate device memory
// themselves or through a library. A host process whose memory is managed by
// its own pooling allocator (so every byte must come from that pool and a
// foreign cudaMalloc would either fail against its reserve or go unaccounted),
// a real-time loop where cudaMalloc/cudaFree would add their host latency and
// cudaFree's implicit device synchronisation to every step, or a plugin that is
// handed pre-allocated buffers and nothing else. bm_area_create allocates the
// slab, the control block, the slice table and the compiled gather offsets;
// this entry point takes the slab from the caller and keeps the rest in one
// file-scope device array that the library holds from load until exit.
//
// The array (kScratchBytes, about 8 MiB) holds, in order: the control block
// (cycle number, device error bits, per-tuft verification status), the slice
// table, and the compiled 16-bit gather offsets of one tuft (kMaxSyns
// synapses). Every call rewrites the control block and the slice table and
// recompiles the gather offsets, so nothing from an earlier call is read.
// Calls share the array: two calls whose work overlaps on the GPU (on
// different streams, or from different threads, on one device) race on it.
#include <cuda.h>

#include <cstring>
#include <mutex>

#include "bm_fused.h"
#include "bm_kernels.h"

using namespace bm;

namespace {

constexpr uint64_t kMaxSyns = 1ull << 22;   // synapses of the largest tuft served (4,194,304)
constexpr size_t kCtlOff = 0;
constexpr size_t kSlicesOff = 1024;
constexpr size_t kGidxOff = 8192;
constexpr size_t kScratchBytes = kGidxOff + kMaxSyns * sizeof(int16_t);
static_assert(sizeof(AreaCtl) <= kSlicesOff - kCtlOff, "control block overlaps the slice table");
static_assert(kSlicesOff + BM_MAX_SLICES * sizeof(SliceRec) <= kGidxOff, "slice table overlaps the offsets");

// In host code this name only stands for the array; its device address comes
// from cudaGetSymbolAddress (scratch_on below).
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct ScratchAddr {
    unsigned char* ptr = nullptr;   // device address of g_scratch
    unsigned long long ctx = 0;     // id of the context it was looked up in
};
ScratchAddr g_scratch_dev[kMaxDevices];   // per device

// Id of the calling thread's current context (cuCtxGetId: unique for the
// life of the process, so a context created after a device reset has a new
// one), or 0 when there is none or the driver lacks the call. The driver
// entry points are resolved through the runtime, so the library needs no
// link against the driver library.
unsigned long long current_ctx_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool resolved = false;
    if (!resolved) {
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa{}, qb{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &a, 12000, cudaEnableDefault, &qa) == cudaSuccess &&
            cudaGetDriverEntryPointByVersion("cuCtxGetId", &b, 12000, cudaEnableDefault, &qb) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess && qb == cudaDriverEntryPointSuccess) {
            get_current = (GetCurrent)a;
            get_id = (GetId)b;
        }
        cudaGetLastError();
        resolved = true;
    }
    if (!get_current || !get_id) return 0;
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the array on `dev` (the current device). Looked up on the
// first call made with that device current, and again whenever the current
// context is not the one the address was looked up in (a device reset
// replaces the primary context and may move the array).
int scratch_on(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kMaxDevices)
        return set_err(BM_ERR_NO_DEVICE, "bm_tuft_cycle_static: device %d beyond the %d served", dev, kMaxDevices);
    std::lock_guard<std::mutex> g(g_mu);
    ScratchAddr& S = g_scratch_dev[dev];
    const unsigned long long ctx = current_ctx_id();
    if (!S.ptr || !ctx || ctx != S.ctx) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p)
            return set_err(BM_ERR_CUDA, "bm_tuft_cycle_static: cudaGetSymbolAddress of the scratch array on device %d: %s",
                           dev, cudaGetErrorString(e));
        S.ptr = (unsigned char*)p;
        S.ctx = current_ctx_id();   // the lookup made the device's context current if none was
    }
    *out = S.ptr;
    return BM_OK;
}

struct SliceTable {
    SliceRec r[BM_MAX_SLICES];
};

// Control block and slice table of this call, from kernel parameters (no copy).
__global__ void k_static_begin(unsigned char* scratch, const SliceTable tab, unsigned long long cycle) {
    AreaCtl* ctl = (AreaCtl*)(scratch + kCtlOff);
    SliceRec* slices = (SliceRec*)(scratch + kSlicesOff);
    for (uint32_t k = threadIdx.x; k < BM_MAX_SLICES; k += blockDim.x) slices[k] = tab.r[k];
    for (uint32_t k = threadIdx.x; k < BM_MAX_LAYERS * BM_MAX_TUFTS; k += blockDim.x) ctl->tuft_status[k] = 0;
    if (threadIdx.x == 0) {
        ctl->cycle = cycle;
        ctl->error = 0;
        ctl->wait_us = 0;
        ctl->stall_stage = 0;
        ctl->blocks_done = 0;
        ctl->host_err = nullptr;
    }
}

__global__ void k_static_end(const unsigned char* scratch, uint32_t* error_out) {
    *error_out = ((const AreaCtl*)(scratch + kCtlOff))->error;
}

}  // namespace

extern "C" int bm_tuft_cycle_static(const bm_area_plan* plan, uint32_t layer, uint32_t tuft, void* slab,
                                    uint64_t cycle, uint32_t* dev_error_out, void* stream) {
    if (!plan || !slab) return set_err(BM_ERR_INVALID, "bm_tuft_cycle_static: null plan or slab");
    const bm_area_plan& P = *plan;
    if (P.n_layers > BM_MAX_LAYERS || P.n_slices > BM_MAX_SLICES)
        return set_err(BM_ERR_INVALID, "bm_tuft_cycle_static: malformed plan (%u layers, %u slices)", P.n_layers,
                       P.n_slices);
    if (layer >= P.n_layers)
        return set_err(BM_ERR_INVALID, "bm_tuft_cycle_static: layer %u out of range (%u data layers)", layer,
                       P.n_layers);
    const bm_layer_plan& L = P.layers[layer];
    if (tuft >= L.n_tufts || tuft >= BM_MAX_TUFTS)
        return set_err(BM_ERR_INVALID, "bm_tuft_cycle_static: tuft %u out of range (layer %u has %u)", tuft, layer,
                       L.n_tufts);
    const uint64_t n_syn = (uint64_t)L.cells * L.tufts[tuft].syns_per_tft;
    if (n_syn > kMaxSyns)
        return set_err(BM_ERR_INVALID,
                       "bm_tuft_cycle_static: tuft %u of layer %u has %llu synapses; the library-held scratch "
                       "serves at most %llu per call",
                       tuft, layer, (unsigned long long)n_syn, (unsigned long long)kMaxSyns);
    // An error the caller's own earlier work left pending is reported, not
    // cleared: the launches below are checked on their own.
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess)
        return set_err(BM_ERR_CUDA, "bm_tuft_cycle_static: a CUDA error was pending before the call: %s",
                       cudaGetErrorString(e));
    int dev = -1;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_err(BM_ERR_NO_DEVICE, "bm_tuft_cycle_static: no CUDA device (%s)", cudaGetErrorString(e));
    unsigned char* scratch = nullptr;
    int rc = scratch_on(dev, &scratch);
    if (rc != BM_OK) return rc;

    if ((uintptr_t)slab & 255)
        return set_err(BM_ERR_INVALID, "bm_tuft_cycle_static: the slab must be 256-byte aligned (as cudaMalloc returns)");
    FusedArea F;
    plan_fused_tuft(F, P, layer, tuft);
    bind_fused_tuft(F, P, layer, tuft, (const uint8_t*)slab + P.axon_off);
    FusedTuft& FT = F.t[layer][tuft];
    if (!FT.ok)
        return set_err(BM_ERR_UNSUPPORTED,
                       "bm_tuft_cycle_static: tuft %u of layer %u is outside the fused kernel's shapes "
                       "(syns_per_den a power of two in 16..512, dens_per_tft a power of two, 16-byte aligned buffers)",
                       tuft, layer);
    if (FT.tiled) FT.gidx = (uint16_t*)(scratch + kGidxOff);
    DevLayer D;
    fill_dev_layer(D, P, layer, (uint8_t*)slab);
    SliceTable tab;
    fill_slice_table(P, tab.r);

    cudaStream_t s = (cudaStream_t)stream;
    AreaCtl* ctl = (AreaCtl*)(scratch + kCtlOff);
    const SliceRec* slices = (const SliceRec*)(scratch + kSlicesOff);
    k_static_begin<<<1, 256, 0, s>>>(scratch, tab, (unsigned long long)cycle);
    launch_compile_tuft(F, D, layer, tuft, ctl, s);
    launch_fused_tuft(F, (const uint8_t*)slab + P.axon_off, slices, D, layer, tuft, ctl, s);
    if (dev_error_out) k_static_end<<<1, 1, 0, s>>>(scratch, dev_error_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_err(BM_ERR_CUDA, "bm_tuft_cycle_static: launch failed: %s", cudaGetErrorString(e));
    return BM_OK;
}
