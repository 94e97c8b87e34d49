// bm_dev.cuh -- device-side data structures and integer helpers shared by the
// cycle kernels. Every helper states the bismit OpenCL function it restates
// (paths relative to the bismit repository).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/bismit_b200.h"

#include <utility>

namespace bm {

// Programmatic dependent launch. The cycle's kernels are launched with the
// programmatic-serialization attribute (launch_pdl), so a kernel's blocks may
// be scheduled while the previous kernel of the stream drains. Every such
// kernel calls pdl_begin() before touching global memory: it waits until the
// previous kernel has finished and its writes are visible, then lets the next
// kernel be scheduled. Launched without the attribute, both are no-ops.
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// Reference constants: cl/bismit.cl:11-22, cl/control.cl:6-13,
// src/cmn/mod.rs:242,321-336.
constexpr int kSynapseAxonBiasLog2 = 1;
constexpr int kDendriteActivityDecay = 1536;
constexpr int kCellActivityDecay = 768;
constexpr int kInhibCenterOffset = 1;
constexpr int kInhibHorizOffset = 3;
constexpr int kSlcSclCoeffL2 = 4;
constexpr int kRetinalThreshold = 48;   // RETNAL_THRESHOLD, cl/bismit.cl:19
constexpr uint8_t kCelPrevActiveFlag = 0x08;
constexpr uint8_t kSynPrevActiveFlag = 0x10;
constexpr uint32_t kDenBasalProximalFlag = 0x01;
constexpr uint32_t kDenBasalDistalFlag = 0x02;

// One slice of the area's axon space, packed for a single 16-byte load:
// x = first axon (axn_slc_idzs), y = v_size | u_size << 16,
// z = v_scale | u_scale << 8 | v_mid << 16 | u_mid << 24.
typedef uint4 SliceRec;

struct DevTuft {
    uint32_t dpt, spd, spt, mad_l2, thresh, den_kind;
    uint64_t syn_idz, den_idz, cel_idz;
    uint64_t rnd_key_den;   // den_cycle_tft per-launch value key
    uint64_t rnd_key_mtp;   // tft_dst_mtp per-launch value key
};

struct DevLayer {
    uint32_t kind, depth, v_size, u_size, cells, base_slc, axn_idz, n_tufts;
    uint32_t enabled_flags, prx_id, dst_id, apc_id;
    uint64_t n_syns;
    uint8_t* buf[BM_BUF_COUNT];
    DevTuft tft[BM_MAX_TUFTS];
    uint64_t rnd_key_ssc_mtp;
};

// Per-area control block in device memory.
// Device-side error bits (AreaCtl::error).
constexpr unsigned int kErrWaitTimeout = 1u;   // a bounded mbarrier wait gave up

// Tuft status bits (AreaCtl::tuft_status), written by the source verifier.
constexpr unsigned int kTuftSrcOutsideTile = 1u;   // some source is not served by the staged tile
constexpr unsigned int kTuftFlagsForeign = 2u;     // some flag byte has bits other than SYN_PREV_ACTIVE

struct AreaCtl {
    unsigned long long cycle;       // cycle number of the cycle in flight
    unsigned int error;             // sticky device-side error bits (kErr*)
    unsigned int wait_us;           // limit of each bounded wait in the tuft kernels, us (0: kDefaultWaitUs)
    unsigned int stall_stage;       // fault injection: the stage producer that takes a tuft's first tile
                                    // withholds its stall_stage-th stage from it on (0: none)
    unsigned int blocks_done;       // blocks of a cycle-ending kernel done so far (0 between cycles)
    unsigned int* host_err;         // host-mapped word the cycle end copies non-zero error bits to
                                    // (null: none), so the host sees them without a synchronisation
    unsigned int tuft_status[BM_MAX_LAYERS * BM_MAX_TUFTS];
};
constexpr unsigned int kDefaultWaitUs = 2000000u;   // 2 s

// The cycle's last kernel: advance the counter, and mirror any error bits to
// the host-mapped word.
__device__ __forceinline__ void end_cycle(AreaCtl* c) {
    c->cycle += 1;
    const unsigned int e = c->error;
    if (e && c->host_err) *(volatile unsigned int*)c->host_err = e;
}

__host__ __device__ inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// The per-launch random value for a (layer, role, tuft) key at `cycle`:
// key = splitmix64(splitmix64(seed) + bits) is precomputed on the host.
__host__ __device__ inline int32_t rnd_at(uint64_t key, uint64_t cycle) {
    return (int32_t)(uint32_t)(splitmix64(key + cycle) >> 32);
}

__device__ __forceinline__ int32_t shl32(int32_t x, int n) { return (int32_t)((uint32_t)x << n); }

// rnd_mix, cl/bismit.cl:426-431 (>> on a signed int is arithmetic in CUDA).
__device__ __forceinline__ int32_t rnd_mix(int32_t rnd_a, int32_t seed) {
    seed ^= shl32(seed ^ rnd_a, 13);
    seed ^= seed >> 17;
    seed ^= shl32(seed, 5);
    return seed;
}

// rnd_inc / rnd_dec, cl/bismit.cl:447-469.
__device__ __forceinline__ int rnd_inc(int32_t rnd_a, int32_t seed, int8_t val, int32_t mask) {
    int a = val < 0 ? -(int)val : (int)val;
    return (rnd_mix(rnd_a, seed) & mask) > (a + (mask - 0x7f));
}
__device__ __forceinline__ int rnd_dec(int32_t rnd_a, int32_t seed, int8_t val, int32_t mask) {
    int a = val < 0 ? -(int)val : (int)val;
    return (rnd_mix(rnd_a, seed) & mask) > ((a - (val == 127)) + (mask - 0x7f));
}

// update_activity_rating, cl/bismit.cl:531-540 (rnd_inc_u :482-484, rnd_0xFFFF :525-527).
__device__ __forceinline__ uint8_t update_activity(uint8_t act, int is_active, int32_t rnd, int32_t seed,
                                                   int decay) {
    act = (uint8_t)(act + (((rnd_mix(rnd, seed) & 0xFF) > act) & is_active));
    act = (uint8_t)(act - (((rnd_mix(rnd, shl32(seed, 1)) & 0xFFFF) < decay) & (act > 0)));
    return act;
}

// syn_fire, cl/syns.cl:2-4.
__device__ __forceinline__ uint8_t syn_fire(uint8_t a) {
    return (uint8_t)(((a != 0) << 7) + (a >> kSynapseAxonBiasLog2));
}

// axn_idx_3d_unsafe (cl/bismit.cl:323-363, scalar: the slice mid is added to
// the i8 offset in an i8) and its vec4 form (:366-391: added in int).
__device__ __forceinline__ uint32_t axn_idx(const SliceRec& s, uint32_t v_id, int v_ofs8, uint32_t u_id,
                                            int u_ofs8, bool vec4, bool& safe) {
    int v_size = (int)(s.y & 0xFFFF), u_size = (int)(s.y >> 16);
    int v_mid = (int)((s.z >> 16) & 0xFF), u_mid = (int)(s.z >> 24);
    int v_ofs = v_ofs8 + v_mid, u_ofs = u_ofs8 + u_mid;
    if (!vec4) {
        v_ofs = (int)(int8_t)(uint8_t)v_ofs;
        u_ofs = (int)(int8_t)(uint8_t)u_ofs;
    }
    int v_sc = (int)((v_id * (s.z & 0xFF)) >> kSlcSclCoeffL2);
    int u_sc = (int)((u_id * ((s.z >> 8) & 0xFF)) >> kSlcSclCoeffL2);
    int vt = v_sc + v_ofs, ut = u_sc + u_ofs;
    safe = (vt >= 0) & (vt < v_size) & (ut >= 0) & (ut < u_size);
    return s.x + (uint32_t)(vt * u_size + ut);
}

}  // namespace bm
