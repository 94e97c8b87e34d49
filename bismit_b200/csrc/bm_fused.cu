// bm_fused.cu -- fused stage kernels.
//
// fused_tuft_cycle: for one tuft of one layer, in a single pass over its
// synapses, does what bismit runs as four launches:
//   tft_set_syn_flags          cl/syns.cl:23-33
//   layer_cycle_syns_wow[_vec4] cl/syns.cl:179-388
//   den_cycle_tft               cl/bismit.cl:695-747
//   tft_cycle (pyramidal)       cl/bismit.cl:755-842
// The flags kernel runs over every tuft of the layer before any synapse
// kernel; the flags of a tuft depend only on that tuft's states, which only its
// own synapse kernel writes, so doing both per tuft is equivalent.
//
// Main form (k_fused_tuft_tma), for tufts whose source slices share one
// geometry: persistent CTAs of 8 consumer warps and 1 producer warp walk tiles
// of cells (part of a row, or whole rows, of one layer slice).
//  * Per tile the consumers stage the axon footprint the tile's synapses can
//    reach -- the tile's scaled extent plus the pool's largest offsets, for
//    every source slice -- in shared memory as already-fired synapse states
//    (syn_fire(axon), 0 outside the slice).
//  * The producer warp streams the tile's synapse arrays into a ring of
//    shared-memory stages with TMA bulk copies (cp.async.bulk) that complete
//    on mbarriers, running up to NST stages ahead of the consumers.
//  * A consumer warp takes 512 synapses of a stage (32 lanes x 16), computes
//    new states and flags, writes them with 16-byte stores, reduces dendrite
//    sums across syns_per_den/16 lanes with shuffles and the tuft argmax across
//    the cell's lanes (redux.sync over the warp when a cell fills it).
//
// Gather index: each synapse's (source slice, v offset, u offset) is compiled
// once into a 16-bit offset into the staged footprint, (slc - slc0) * TSZ +
// v_ofs * TW + u_ofs, kept beside the synapse arrays (the canonical source
// arrays are unchanged and remain what readback returns). The compile pass
// runs at build and again whenever the caller writes sources or flags. A
// source it cannot express (slice outside the pool, offset beyond the pool's
// reach -- only possible through caller writes) marks the tuft, and the
// kernel then streams the original arrays and indexes every synapse as
// axn_state_3d_safe (cl/bismit.cl:397-418) does.
//
// Every mbarrier wait is bounded; on a timeout the kernel records
// kErrWaitTimeout, lets its own copies in flight land and returns.
#include "bm_fused.h"

#include <cuda.h>

#include <algorithm>
#include <cstddef>
#include <cstring>
#include <new>

#include "bm_kernels.h"

namespace bm {

namespace {

constexpr int kWarps = 8;                    // consumer warps per CTA (tiled form)
constexpr int kThreads = (kWarps + 1) * 32;  // plus one producer warp
constexpr int kMaxRecs = 8;                  // contiguous source slices served by the fast gathers
constexpr uint32_t kMaxSmem = 110 * 1024;    // dynamic shared memory per CTA (two CTAs per SM)
constexpr uint32_t kSmem3 = 73 * 1024;       // ... with which three CTAs fit one SM
constexpr uint32_t kWaitLimit = 1u << 22;

struct FusedTuftArgs {
    CUtensorMap tmap;       // footprint box of the recorded slices (fp_tma); first, for its 64-byte alignment
    const uint8_t* axns;
    const SliceRec* slices;
    AreaCtl* ctl;
    const uint8_t* slc;     // tuft-relative synapse arrays
    const int8_t* vofs;
    const int8_t* uofs;
    const int8_t* str;
    uint8_t* st;
    uint8_t* fl;
    const uint16_t* gidx;   // compiled gather offsets (tiled form): bytes into the tile's footprint
    uint8_t* den_act;       // tuft-relative dendrite arrays
    uint8_t* den_raw;
    uint8_t* den_st;
    uint8_t* cel_en;        // spiny stellate cell energies (ssc_soma)
    uint8_t* t_pid;         // tuft-relative cell-tuft arrays (pyramidal)
    uint8_t* t_praw;
    uint8_t* t_pst;
    uint8_t* t_ptft;
    uint8_t* t_bid;
    uint8_t* t_braw;
    uint8_t* t_bst;
    uint8_t* t_st;
    uint64_t n_syn;         // synapses in the tuft
    uint32_t den_idz;       // first dendrite (layer index) for the activity seed
    uint32_t thresh;
    uint32_t cols, u_size, v_size;
    uint32_t S_l2, spd_l2, lpd_l2, lpc_l2;   // log2: syns/cell-tuft, syns/den, lanes/den, lanes/cell (<= 5)
    uint32_t chunks_per_unit;
    uint32_t mad_l2;
    uint32_t slc0, nrec;    // fast gathers serve slice ids slc0 .. slc0 + nrec - 1
    uint32_t vec4;          // bismit's vec4 synapse kernel semantics (spt % 4 == 0)
    uint64_t rnd_key;
    uint32_t status_idx;    // index into AreaCtl::tuft_status
    // Global-record form: units are chunks (S <= 512) or cells (S > 512).
    uint64_t n_units;
    // Tiled form.
    uint32_t tile_w, tile_h, tiles_u, tiles_v, n_tiles;
    uint64_t usz_magic;                 // div_magic(u_size), for multi-row tiles
    uint64_t per_slice_magic, tiles_u_magic;   // div_magic of the tiles per slice and per row
    int32_t rv, ru;                     // largest |v|, |u| offset served from the footprint
    uint32_t fw, frows, fsz;            // footprint width, rows and bytes per source slice
    uint32_t src_vs, src_us, src_vsz, src_usz;   // geometry shared by the recorded slices
    uint32_t src_idz[kMaxRecs];
    uint32_t nst;                       // pipeline stages
    uint32_t stage_bytes;               // bytes per 1-byte array per stage
    uint32_t ring_off;                  // byte offset of the ring (mbarriers, then stages) in dynamic smem;
                                        // the footprint starts at 0
    uint32_t unit_l2;                   // log2 of the bytes of one unit (chunks_per_unit * 512)
    uint32_t stage_stride;              // bytes per ring buffer (synapse arrays + windows)
    uint32_t win;                       // dendrite / cell-tuft windows ride in the stages
    uint32_t win_bytes;                 // bytes per window
    uint32_t geom;                      // specialised consumer for this shape (0: the general one)
    uint32_t fp_tma;                    // the footprint comes from a tensor box load (else consumers stage it)
    uint32_t ssc_soma;                  // also run ssc_cycle (spiny stellate cells of one dendrite)
    uint32_t fp_bytes;                  // bytes of that box (nrec * frows * fw)
    uint32_t cycle_from_host;           // take the cycle number from `cycle` rather than the area's counter
    unsigned long long cycle;           // (a launch on the area's front stream, which may run ahead of the
                                        // counter: the host knows the number of the cycle it enqueues)
};
// The cycle number a launch draws its random value for.
__device__ __forceinline__ unsigned long long cycle_of(const FusedTuftArgs& A) {
    return A.cycle_from_host ? A.cycle : A.ctl->cycle;
}
static_assert(offsetof(FusedTuftArgs, tmap) == 0 && alignof(FusedTuftArgs) >= 64,
              "the tensor map must sit 64-byte aligned in the parameter block");

// Lanes of a cell write its eight cell-tuft fields through one pointer table.
static_assert(offsetof(FusedTuftArgs, t_st) == offsetof(FusedTuftArgs, t_pid) + 7 * sizeof(uint8_t*),
              "the cell-tuft arrays must be consecutive pointers");

struct Rec {
    int32_t base;     // idz + vsc * u_size + usc
    int32_t vsc, usc; // scaled position plus mid
    uint32_t dims;    // v_size | u_size << 16
};

// ---------------------------------------------------------------- PTX ----
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t tx) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(tx) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// try_wait that may suspend the thread until the phase completes, for at most
// `hint_ns` nanoseconds per call (a suspended warp issues nothing).
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: false once `limit_us` microseconds of wall time have passed
// without the phase completing (and in any case after kWaitLimit suspended
// tries).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit_us) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 0; i < kWaitLimit; i++) {
        if (mbar_try_wait_sleep(bar, parity, 200000u)) return true;
        if (global_ns() - t0 > 1000ull * limit_us) return false;
    }
    return false;
}
// The wait limit of an area's tuft launches, us (AreaCtl::wait_us; 0: the
// default).
__device__ __forceinline__ uint32_t wait_limit_us(const AreaCtl* ctl) {
    const unsigned int us = ctl ? ctl->wait_us : 0u;
    return us ? us : kDefaultWaitUs;
}

// A consumer warp's ring position and phases, in one word (it is carried
// across every tile and stage): bits 0-2 the ring buffer, bit 3 the ring's
// phase, bit 4 the footprint box's phase.
constexpr uint32_t kRingBuf = 7u, kRingPhase = 8u, kFpPhase = 16u;
// 1-D bulk copy global -> shared completing on `bar` (16-byte aligned, size % 16 == 0).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
// 3-D tensor box load global -> shared completing on `bar` (no multicast;
// the box's x coordinate is a multiple of 16 bytes, elements outside the
// tensor read as 0).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int32_t x, int32_t y, int32_t z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}
// Orders this thread's generic shared-memory writes before later writes of
// the async proxy (a tensor load into the same bytes).
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// Barrier among the consumer warps only (the producer warp runs free).
__device__ __forceinline__ void consumers_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kWarps * 32) : "memory"); }
// The same barrier, returning the OR of `p` over the consumer warps: every
// consumer thread gets the same answer, so decisions taken on it stay uniform.
__device__ __forceinline__ bool consumers_sync_or(bool p) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred q, o;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "barrier.cta.red.or.pred o, 1, %2, q;\n\t"
        "selp.u32 %0, 1, 0, o;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)p), "n"(kWarps * 32)
        : "memory");
    return r != 0;
}

// ------------------------------------------------------------ helpers ----
// 0xFF in every byte of x whose sign bit is set (prmt's sign-replicate mode).
__device__ __forceinline__ uint32_t sign_bytes(uint32_t x) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, 0xBA98;" : "=r"(r) : "r"(x), "r"(0u));
    return r;
}
// The low bytes of a0..a3 as one word (a0 lowest).
__device__ __forceinline__ uint32_t pack4(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3) {
    return __byte_perm(__byte_perm(a0, a1, 0x0040), __byte_perm(a2, a3, 0x0040), 0x5410);
}
__device__ __forceinline__ uint32_t nz_bits(uint32_t x) {
    // 0x80 in every byte of x that is non-zero.
    return (((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x) & 0x80808080u;
}

// ssc_cycle (cl/bismit.cl:849-884) folded into the spiny stellate tuft stage
// for cells of one dendrite, whose soma state is that dendrite's state: from
// cell c's energy and the dendrite state just computed, writes the energy and
// returns the soma state.
__device__ __forceinline__ uint32_t ssc_soma(uint8_t* en, uint32_t c, uint32_t energy, uint32_t state) {
    const int active = state != 0;
    const int restless = (energy > 191) & active;
    const int dark = energy == 255;
    en[c] = (uint8_t)((dark | restless) ? energy - 64 : energy);
    return min(state + (uint32_t)restless * 255u + (uint32_t)dark * 255u, 255u);
}

__device__ __forceinline__ uint8_t gather_general(const FusedTuftArgs& A, uint32_t slc, uint32_t v, uint32_t u,
                                                  int vo, int uo) {
    bool safe;
    uint32_t ai = axn_idx(A.slices[slc], v, vo, u, uo, A.vec4 != 0, safe);
    return syn_fire(safe ? __ldg(A.axns + ai) : (uint8_t)0);
}

// Loads issued at the start of a chunk so their latency overlaps the gathers:
// the activity of the lane's dendrite (dendrite-lead lanes) and, at the first
// chunk of a cell, the cell-tuft's current best/state bytes that the tuft
// cycle copies to the prev arrays. Cells of 8 or more lanes spread that copy
// over lanes: lane f < 4 of the cell holds field f (best id, best raw, best
// state, tuft state); smaller cells keep all four, packed, in their first lane.
__device__ __forceinline__ uint32_t prefetch_act(const FusedTuftArgs& A, uint64_t off, bool on, int lane) {
    const uint32_t lpd = 1u << A.lpd_l2;
    return (on && (lane & (lpd - 1)) == 0) ? (uint32_t)A.den_act[off >> A.spd_l2] : 0u;
}
template <bool TUFT>
__device__ __forceinline__ uint32_t prefetch_tuft(const FusedTuftArgs& A, uint64_t off, bool on, int lane) {
    if (!TUFT || !on) return 0u;
    const uint32_t f = lane & ((1u << A.lpc_l2) - 1);
    const uint32_t c = (uint32_t)(off >> A.S_l2);
    if (A.lpc_l2 >= 3) return f < 4 ? (uint32_t)(&A.t_bid)[f][c] : 0u;
    if (f != 0) return 0u;
    return (uint32_t)A.t_bid[c] | ((uint32_t)A.t_braw[c] << 8) | ((uint32_t)A.t_bst[c] << 16) |
           ((uint32_t)A.t_st[c] << 24);
}

// Everything after the new states of 16 synapses are known, for one 512-byte
// chunk: flags, stores, dendrite reductions and the chunk's share of the tuft
// reduction. `last` marks the final chunk of a cell.
template <bool TUFT>
__device__ __forceinline__ void finish_chunk(const FusedTuftArgs& A, const uint4& str4, const uint4& st4,
                                             const uint4& fl4, const uint4& nst4, bool flags_clean, uint32_t off,
                                             bool on, int lane, int32_t rnd, bool last, uint32_t act0,
                                             uint32_t tuft_cur, uint32_t& t_key, uint32_t& t_best, uint32_t& t_sum) {
    const uint32_t lpd = 1u << A.lpd_l2;
    const uint32_t lpc = 1u << A.lpc_l2;
    uint32_t sum = 0, raw = 0;
    if (on) {
        const uint32_t* strw = (const uint32_t*)&str4;
        const uint32_t* stw = (const uint32_t*)&st4;
        const uint32_t* flw = (const uint32_t*)&fl4;
        const uint32_t* nstw = (const uint32_t*)&nst4;
        uint4 nfl4;
        uint32_t* nflw = (uint32_t*)&nfl4;
#pragma unroll
        for (int w = 0; w < 4; w++) {
            const uint32_t keep = flags_clean ? 0u : (flw[w] & 0xEFEFEFEFu);
            nflw[w] = keep | (nz_bits(stw[w]) >> 3);
            raw = __dp4a(nstw[w], 0x01010101u, raw);
            sum = __dp4a(nstw[w] & ~sign_bytes(strw[w]), 0x01010101u, sum);
        }
        *(uint4*)(A.st + off) = nst4;
        *(uint4*)(A.fl + off) = nfl4;
    }
    for (uint32_t m = 1; m < lpd; m <<= 1) {
        sum += __shfl_xor_sync(0xFFFFFFFFu, sum, m);
        raw += __shfl_xor_sync(0xFFFFFFFFu, raw, m);
    }
    uint32_t d_raw = 0, d_st = 0;
    const bool lead = on && (lane & (lpd - 1)) == 0;
    const uint32_t den = off >> A.spd_l2;   // dendrite id within the tuft
    if (lead) {
        const int active = sum > A.thresh;
        const uint32_t s2 = active ? sum : 0u;
        const uint32_t di = den + A.den_idz;
        const uint32_t seed = (raw + A.thresh) | di;
        A.den_act[den] = update_activity((uint8_t)act0, active, rnd, (int32_t)seed, kDendriteActivityDecay);
        d_raw = min(raw >> 4, 255u);
        d_st = min(s2 >> 4, 255u);
        A.den_raw[den] = (uint8_t)d_raw;
        if (!TUFT && A.ssc_soma) d_st = ssc_soma(A.cel_en, den, A.cel_en[den], d_st);
        A.den_st[den] = (uint8_t)d_st;
    }
    if (TUFT) {
        // Argmax of the raw state with the first (lowest) dendrite winning
        // ties: maximise (raw << 16 | (0xFFFF - id)).
        const uint32_t den_in_cell = den & ((1u << (A.S_l2 - A.spd_l2)) - 1);
        uint32_t key = lead ? ((d_raw << 16) | (0xFFFFu - den_in_cell)) : 0u;
        uint32_t best = d_st, tot = d_st;
        if (lpc == 32) {
            key = __reduce_max_sync(0xFFFFFFFFu, key);
            best = __reduce_max_sync(0xFFFFFFFFu, best);
            tot = __reduce_add_sync(0xFFFFFFFFu, tot);
        } else {
            for (uint32_t m = lpd; m < lpc; m <<= 1) {
                key = max(key, __shfl_xor_sync(0xFFFFFFFFu, key, m));
                best = max(best, __shfl_xor_sync(0xFFFFFFFFu, best, m));
                tot += __shfl_xor_sync(0xFFFFFFFFu, tot, m);
            }
            // The butterfly leaves the cell's totals in its dendrite-lead
            // lanes only; every lane of the cell writes a field.
            if (lpd > 1 && lpc >= 8) {
                const int src = lane & ~(int)(lpd - 1);
                key = __shfl_sync(0xFFFFFFFFu, key, src);
                best = __shfl_sync(0xFFFFFFFFu, best, src);
                tot = __shfl_sync(0xFFFFFFFFu, tot, src);
            }
        }
        t_key = max(t_key, key);
        t_best = max(t_best, best);
        t_sum += tot;
        const uint32_t f = lane & (lpc - 1);
        if (last && on && (lpc >= 8 ? f < 8 : f == 0)) {
            const uint32_t c = off >> A.S_l2;
            const uint32_t best_raw = t_key >> 16;
            const uint32_t best_id = best_raw ? (0xFFFFu - (t_key & 0xFFFFu)) : 0u;
            const bool is_max = t_sum >= (1u << (A.mad_l2 + 8));
            const uint32_t tst = is_max ? 255u : ((t_sum >> A.mad_l2) & 0xFFu);
            if (lpc >= 8) {
                // Lane f writes field f: the prev copies of the current fields
                // (f < 4), then best id, best raw, best state, tuft state. The
                // eight arrays are consecutive in the arguments.
                const uint32_t nv = f == 4 ? best_id : f == 5 ? best_raw : f == 6 ? t_best : tst;
                (&A.t_pid)[f][c] = (uint8_t)(f < 4 ? tuft_cur : nv);
            } else {
                A.t_pid[c] = (uint8_t)tuft_cur;
                A.t_praw[c] = (uint8_t)(tuft_cur >> 8);
                A.t_pst[c] = (uint8_t)(tuft_cur >> 16);
                A.t_ptft[c] = (uint8_t)(tuft_cur >> 24);
                A.t_bid[c] = (uint8_t)best_id;
                A.t_braw[c] = (uint8_t)best_raw;
                A.t_bst[c] = (uint8_t)t_best;
                A.t_st[c] = (uint8_t)tst;
            }
        }
    }
}

// ------------------------------------------------ global-record form ----
// For tufts whose source slices do not share one geometry: warps stride over
// units of the whole tuft and gather through per-lane slice records.
template <bool TUFT>
__global__ void __launch_bounds__(kWarps * 32) k_fused_tuft(FusedTuftArgs A) {
    pdl_begin();
    __shared__ Rec recs[kWarps][kMaxRecs * 32];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const uint64_t gwarp = (uint64_t)blockIdx.x * kWarps + wib;
    const uint64_t nwarps = (uint64_t)gridDim.x * kWarps;
    const int32_t rnd = rnd_at(A.rnd_key, cycle_of(A));
    const bool flags_clean = (A.ctl->tuft_status[A.status_idx] & kTuftFlagsForeign) == 0;
    for (uint64_t unit = gwarp; unit < A.n_units; unit += nwarps) {
        uint32_t t_key = 0, t_best = 0, t_sum = 0, tuft_cur = 0;
        for (uint32_t ch = 0; ch < A.chunks_per_unit; ch++) {
            const uint64_t off = (unit * A.chunks_per_unit + ch) * 512 + (uint64_t)lane * 16;
            const bool on = off < A.n_syn;
            const uint32_t cell = (uint32_t)(off >> A.S_l2);
            const uint32_t rem = cell % A.cols;
            const uint32_t v = rem / A.u_size, u = rem % A.u_size;
            __syncwarp();
            for (uint32_t k = 0; k < A.nrec; k++) {
                SliceRec s = A.slices[A.slc0 + k];
                Rec r;
                r.vsc = (int32_t)((v * (s.z & 0xFF)) >> kSlcSclCoeffL2);
                r.usc = (int32_t)((u * ((s.z >> 8) & 0xFF)) >> kSlcSclCoeffL2);
                r.dims = s.y;
                r.base = (int32_t)s.x + r.vsc * (int32_t)(s.y >> 16) + r.usc;
                recs[wib][k * 32 + lane] = r;
            }
            __syncwarp();
            const uint32_t act0 = prefetch_act(A, off, on, lane);
            if (ch == 0) tuft_cur = prefetch_tuft<TUFT>(A, off, on, lane);
            uint4 str4{}, st4{}, fl4{}, nst4{};
            if (on) {
                const uint4 slc4 = __ldg((const uint4*)(A.slc + off));
                const uint4 vo4 = __ldg((const uint4*)(A.vofs + off));
                const uint4 uo4 = __ldg((const uint4*)(A.uofs + off));
                str4 = __ldg((const uint4*)(A.str + off));
                st4 = *(const uint4*)(A.st + off);
                fl4 = *(const uint4*)(A.fl + off);
                const uint32_t* sw = (const uint32_t*)&slc4;
                const uint32_t* vw = (const uint32_t*)&vo4;
                const uint32_t* uw = (const uint32_t*)&uo4;
                uint32_t* ow = (uint32_t*)&nst4;
#pragma unroll
                for (int w = 0; w < 4; w++) {
                    uint32_t out = 0;
#pragma unroll
                    for (int b = 0; b < 4; b++) {
                        const uint32_t slc = (sw[w] >> (8 * b)) & 0xFF;
                        const int vo = (int)(int8_t)(vw[w] >> (8 * b));
                        const int uo = (int)(int8_t)(uw[w] >> (8 * b));
                        const uint32_t k = slc - A.slc0;
                        uint32_t a;
                        if (k < A.nrec) {
                            const Rec r = recs[wib][k * 32 + lane];
                            const int vt = r.vsc + vo, ut = r.usc + uo;
                            const bool safe = ((uint32_t)vt < (r.dims & 0xFFFF)) & ((uint32_t)ut < (r.dims >> 16));
                            a = syn_fire(safe ? __ldg(A.axns + (uint32_t)(r.base + vo * (int32_t)(r.dims >> 16) + uo))
                                              : (uint8_t)0);
                        } else {
                            a = gather_general(A, slc, v, u, vo, uo);
                        }
                        out |= a << (8 * b);
                    }
                    ow[w] = out;
                }
            }
            finish_chunk<TUFT>(A, str4, st4, fl4, nst4, flags_clean, (uint32_t)off, on, lane, rnd,
                               ch + 1 == A.chunks_per_unit, act0, tuft_cur, t_key, t_best, t_sum);
        }
    }
}

// ------------------------------------------------------ tiled TMA form ----
// x / d by a 64-bit multiply-high with m = div_magic(d) = ceil(2^64 / d):
// exact for every 32-bit x and 2 <= d < 2^32 (the rounding error of m
// stays below 2^-32 < 1/d); d == 1 is passed through.
inline uint64_t div_magic(uint32_t d) { return d > 1 ? UINT64_MAX / d + 1 : 0; }
__device__ __forceinline__ uint32_t fast_div(uint32_t x, uint32_t d, uint64_t m) {
    return d == 1 ? x : (uint32_t)__umul64hi((uint64_t)x, m);
}

struct TileGeo {
    uint32_t v0, u0, h, w;
    int32_t vlo, ulo;
    uint32_t xoff;                   // fp_tma: columns sit (ulo & 15) bytes into each footprint row
    uint32_t cell0, syn0, syn_end;   // tuft-relative (a tuft has fewer than 2^32 synapses)
};

__device__ __forceinline__ TileGeo tile_geo(const FusedTuftArgs& A, uint32_t t) {
    TileGeo g;
    const uint32_t per_slice = A.tiles_v * A.tiles_u;
    const uint32_t s_lyr = fast_div(t, per_slice, A.per_slice_magic);
    const uint32_t tr = t - s_lyr * per_slice;
    const uint32_t tv = fast_div(tr, A.tiles_u, A.tiles_u_magic);
    g.v0 = tv * A.tile_h;
    g.u0 = (tr - tv * A.tiles_u) * A.tile_w;
    g.h = min(A.tile_h, A.v_size - g.v0);
    g.w = min(A.tile_w, A.u_size - g.u0);
    g.vlo = (int32_t)((g.v0 * A.src_vs) >> kSlcSclCoeffL2) - A.rv;
    g.ulo = (int32_t)((g.u0 * A.src_us) >> kSlcSclCoeffL2) - A.ru;
    g.xoff = A.fp_tma ? ((uint32_t)g.ulo & 15u) : 0u;
    g.cell0 = s_lyr * A.cols + g.v0 * A.u_size + g.u0;
    g.syn0 = g.cell0 << A.S_l2;
    g.syn_end = (g.cell0 + g.h * g.w) << A.S_l2;
    return g;
}

// The position of the 16 synapses at tuft offset `off` in the footprint of
// tile G: (cell's scaled row - vlo) * fw + (cell's scaled column - ulo).
__device__ __forceinline__ int32_t footprint_base(const FusedTuftArgs& A, const TileGeo& G, uint32_t off,
                                                  uint32_t& v, uint32_t& u) {
    const uint32_t local = (off >> A.S_l2) - G.cell0;
    if (A.tile_h == 1) {
        v = G.v0;
        u = G.u0 + local;
    } else {
        const uint32_t q = fast_div(local, A.u_size, A.usz_magic);
        v = G.v0 + q;
        u = local - q * A.u_size;
    }
    return ((int32_t)((v * A.src_vs) >> kSlcSclCoeffL2) - G.vlo) * (int32_t)A.fw +
           ((int32_t)((u * A.src_us) >> kSlcSclCoeffL2) - G.ulo) + (int32_t)G.xoff;
}

// syn_fire of four packed axon bytes (cl/syns.cl:2-4).
__device__ __forceinline__ uint32_t fire4(uint32_t x) { return nz_bits(x) | ((x >> 1) & 0x7F7F7F7Fu); }

// A footprint the tensor load brought in holds raw axon bytes: fire them in
// place (consumer threads, 16 bytes each per step; the box is a multiple of
// 16 bytes).
__device__ __forceinline__ void fire_footprint(uint8_t* halo, uint32_t bytes) {
    for (uint32_t i = threadIdx.x * 16u; i < bytes; i += kWarps * 32 * 16) {
        uint4 v = *(const uint4*)(halo + i);
        v.x = fire4(v.x);
        v.y = fire4(v.y);
        v.z = fire4(v.z);
        v.w = fire4(v.w);
        *(uint4*)(halo + i) = v;
    }
}

// Stages the tile's footprint: element (k, row, column), row-major, holds
// syn_fire(axon) at (vlo + row, ulo + column) of recorded slice k, or 0
// outside it. Warps take whole rows (warp w: rows w, w + 8, ... of each
// slice); lanes take columns, so loads of a row are coalesced and the four
// loads of a lane are issued before any store.
__device__ __forceinline__ void build_footprint(const FusedTuftArgs& A, const TileGeo& G, uint8_t* halo, int lane,
                                                int wib) {
    for (uint32_t k = 0; k < A.nrec; k++) {
        const uint8_t* slice = A.axns + A.src_idz[k];
        uint8_t* dst_k = halo + k * A.fsz;
        for (uint32_t r = (uint32_t)wib; r < A.frows; r += kWarps) {
            const int32_t vr = G.vlo + (int32_t)r;
            const bool row_in = (uint32_t)vr < A.src_vsz;
            const uint8_t* src = slice + (row_in ? (uint32_t)vr * A.src_usz : 0u);
            uint8_t* dst = dst_k + r * A.fw;
            for (uint32_t c0 = 0; c0 < A.fw; c0 += 128) {
                uint32_t v[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const uint32_t c = c0 + (uint32_t)lane + 32u * q;
                    const int32_t uc = G.ulo + (int32_t)c;
                    v[q] = (row_in && c < A.fw && (uint32_t)uc < A.src_usz) ? (uint32_t)__ldg(src + uc) : 0u;
                }
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const uint32_t c = c0 + (uint32_t)lane + 32u * q;
                    if (c < A.fw) dst[c] = syn_fire((uint8_t)v[q]);
                }
            }
        }
    }
}

// Stage layout, per buffer of 4 x SB bytes of synapse arrays followed by the
// windows: MODE 0 streams gidx (2 bytes a synapse) then strength, state and
// (unless FCLEAN) flags; MODE 1 streams slc, v_ofs, u_ofs, strength, state,
// flags. The common form (MODE 0, FCLEAN) takes SB synapses a stage; the wider
// forms take SB / 2, so every form fits the same buffer.
template <int MODE, bool FCLEAN>
__device__ __forceinline__ uint32_t stage_syns(uint32_t SB) {
    return (MODE == 0 && FCLEAN) ? SB : SB / 2;
}
template <int MODE>
__device__ __forceinline__ uint32_t arr_off(int which, uint32_t SB) {
    // which: 0 strength, 1 state, 2 flags
    return MODE == 0 ? (2 + which) * SB : (3 + which) * SB;
}

// Consumer work of one stage: this warp's unit (a chunk, or a cell of
// chunks_per_unit chunks).
template <bool TUFT, int MODE, bool FCLEAN>
__device__ __forceinline__ void tma_stage(const FusedTuftArgs& A, const TileGeo& G, const uint8_t* halo,
                                          const uint8_t* sb, uint32_t pos, uint32_t n_units_tile, int lane, int wib,
                                          int32_t rnd) {
    const uint32_t SB = stage_syns<MODE, FCLEAN>(A.stage_bytes);   // synapses of this stage's arrays
    const uint32_t cpu = A.chunks_per_unit;
    if ((uint32_t)wib * cpu * 512 >= SB) return;   // half-size stages keep half the warps busy
    const uint32_t unit = ((pos - G.syn0) >> A.unit_l2) + (uint32_t)wib;
    if (unit >= n_units_tile) return;
    uint32_t t_key = 0, t_best = 0, t_sum = 0, tuft_cur = 0;
    for (uint32_t ch = 0; ch < cpu; ch++) {
        const uint32_t so = ((uint32_t)wib * cpu + ch) * 512 + (uint32_t)lane * 16;   // offset within the stage
        const uint32_t off = pos + so;
        const bool on = off < G.syn_end;
        // The general gather form indexes from the cell's footprint position.
        uint32_t v = 0, u = 0;
        int32_t base = 0;
        if (MODE != 0) base = footprint_base(A, G, off, v, u);
        uint32_t act0;
        if (A.win) {
            // The stage carries the dendrite and cell-tuft bytes (windows start
            // at the stage's first dendrite / cell rounded down to 16).
            const uint8_t* wd = sb + 4 * A.stage_bytes;
            const uint32_t lpd = 1u << A.lpd_l2;
            act0 = (on && (lane & (lpd - 1)) == 0) ? (uint32_t)wd[(off >> A.spd_l2) - ((pos >> A.spd_l2) & ~15u)] : 0u;
            if (TUFT && ch == 0) {
                const uint32_t f = lane & ((1u << A.lpc_l2) - 1);
                const uint32_t ci = (off >> A.S_l2) - ((pos >> A.S_l2) & ~15u);
                tuft_cur = 0;
                if (A.lpc_l2 >= 3) {
                    if (on && f < 4) tuft_cur = wd[(1 + f) * A.win_bytes + ci];
                } else if (on && f == 0) {
                    tuft_cur = (uint32_t)wd[A.win_bytes + ci] | ((uint32_t)wd[2 * A.win_bytes + ci] << 8) |
                               ((uint32_t)wd[3 * A.win_bytes + ci] << 16) | ((uint32_t)wd[4 * A.win_bytes + ci] << 24);
                }
            }
        } else {
            act0 = prefetch_act(A, off, on, lane);
            if (ch == 0) tuft_cur = prefetch_tuft<TUFT>(A, off, on, lane);
        }
        uint4 str4{}, st4{}, fl4{}, nst4{};
        if (on) {
            str4 = *(const uint4*)(sb + arr_off<MODE>(0, SB) + so);
            st4 = *(const uint4*)(sb + arr_off<MODE>(1, SB) + so);
            if (!FCLEAN) fl4 = *(const uint4*)(sb + arr_off<MODE>(2, SB) + so);
            uint32_t* ow = (uint32_t*)&nst4;
            if (MODE == 0) {
                // Compiled offsets index the footprint directly (it starts at
                // shared offset 0); the 15-bit mask keeps even a stray offset
                // inside the CTA's shared memory.
                const uint4 g0 = *(const uint4*)(sb + 2 * so);
                const uint4 g1 = *(const uint4*)(sb + 2 * so + 16);
                const uint32_t gw[8] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w};
#pragma unroll
                for (int w = 0; w < 4; w++) {
                    const uint32_t lo = gw[2 * w], hi = gw[2 * w + 1];
                    ow[w] = pack4(halo[lo & 0x7FFFu], halo[(lo >> 16) & 0x7FFFu], halo[hi & 0x7FFFu],
                                  halo[(hi >> 16) & 0x7FFFu]);
                }
            } else {
                const uint4 slc4 = *(const uint4*)(sb + so);
                const uint4 vo4 = *(const uint4*)(sb + SB + so);
                const uint4 uo4 = *(const uint4*)(sb + 2 * SB + so);
                const uint32_t* sw = (const uint32_t*)&slc4;
                const uint32_t* vw = (const uint32_t*)&vo4;
                const uint32_t* uw = (const uint32_t*)&uo4;
#pragma unroll
                for (int w = 0; w < 4; w++) {
                    uint32_t out = 0;
#pragma unroll
                    for (int b = 0; b < 4; b++) {
                        const uint32_t slc = (sw[w] >> (8 * b)) & 0xFF;
                        const int vo = (int)(int8_t)(vw[w] >> (8 * b));
                        const int uo = (int)(int8_t)(uw[w] >> (8 * b));
                        const uint32_t k = slc - A.slc0;
                        const bool in = (k < A.nrec) & ((uint32_t)(vo + A.rv) <= (uint32_t)(2 * A.rv)) &
                                        ((uint32_t)(uo + A.ru) <= (uint32_t)(2 * A.ru));
                        uint32_t a;
                        if (in) a = halo[k * A.fsz + (uint32_t)(base + vo * (int32_t)A.fw + uo)];
                        else a = gather_general(A, slc, v, u, vo, uo);
                        out |= a << (8 * b);
                    }
                    ow[w] = out;
                }
            }
        }
        finish_chunk<TUFT>(A, str4, st4, fl4, nst4, FCLEAN, off, on, lane, rnd, ch + 1 == cpu, act0, tuft_cur, t_key,
                           t_best, t_sum);
    }
}

// ----------------------------------------------------------- fast form ----
// The common case with its shape fixed at compile time: compiled gather
// offsets, flags carrying only SYN_PREV_ACTIVE, cells of at most 512 synapses
// (a warp's 512-synapse unit holds whole cells) and dendrite / cell-tuft
// windows riding in the stages. Dendrites of 2^SPD_L2 synapses span
// LPD = 2^(SPD_L2 - 4) lanes, cells LPC = 2^LPC_L2 lanes. It computes what
// tma_stage + finish_chunk compute for that case, with every loop bound,
// shift and branch on the shape resolved by the compiler.
// Shapes: 1 (spd 32, S 32), 2 (64, 64), 3 (16, 128), 4 (16, 256), 5 (32, 256),
// 6 (32, 512), 7 (64, 512), 8 (64, 1024: a warp takes a cell in two halves).
constexpr int kGeoms = 9;
__host__ __device__ constexpr int geom_spd_l2(int g) {
    return g == 1 ? 5 : g == 2 ? 6 : g == 3 ? 4 : g == 4 ? 4 : g == 5 ? 5 : g == 6 ? 5 : 6;
}
__host__ __device__ constexpr int geom_lpc_l2(int g) {
    return g == 1 ? 1 : g == 2 ? 2 : g == 3 ? 3 : g == 4 ? 4 : g == 5 ? 4 : g == 8 ? 6 : 5;
}

}  // namespace

// The specialised consumer a tiled tuft's launches dispatch to: shapes 3..7
// on pyramidal layers, 1..2 on spiny stellate layers, 0 (the general
// consumer) otherwise. It applies while the tuft's flags are clean and its
// sources lie in the footprint.
uint32_t consumer_shape(const FusedTuft& FT, uint32_t spt, uint32_t spd, bool pyramidal) {
    if (!FT.tiled || !FT.win || spt > 1024 || FT.stage_bytes != (uint32_t)kWarps * 512 * (spt > 512 ? spt / 512 : 1))
        return 0;
    for (int g = 1; g < kGeoms; g++)
        if ((1u << geom_spd_l2(g)) == spd && (1u << (geom_lpc_l2(g) + 4)) == spt)
            return (pyramidal ? g >= 3 : g <= 2) ? (uint32_t)g : 0u;
    return 0;
}

namespace {

template <bool TUFT, int SPD_L2, int LPC_L2>
__device__ __forceinline__ void stage_fast(const FusedTuftArgs& A, const TileGeo& G, const uint8_t* halo,
                                           const uint8_t* sb, uint32_t pos, int lane, int wib, int32_t rnd) {
    // A cell of 1024 synapses (LPC_L2 == 6) is one warp's unit, taken as two
    // halves of 512 synapses whose per-lane tuft reductions combine before
    // the warp's; its stages hold kWarps such cells (the general consumer's
    // layout for cells above 512 synapses).
    constexpr uint32_t HALVES = LPC_L2 == 6 ? 2u : 1u;
    constexpr uint32_t UNIT = 512u * HALVES;             // synapses of a warp per stage
    constexpr uint32_t SB = kWarps * UNIT;
    constexpr uint32_t WIN = SB / 16 + 32;
    constexpr uint32_t LPD = 1u << (SPD_L2 - 4);
    constexpr uint32_t LPC = 1u << LPC_L2;               // lanes a cell spans over its halves
    constexpr uint32_t LPCW = LPC > 32 ? 32u : LPC;      // lanes of a cell within one half
    constexpr uint32_t S_L2 = LPC_L2 + 4;
    static_assert(LPC >= LPD, "a cell holds whole dendrites");
    const uint32_t unit0 = pos + (uint32_t)wib * UNIT;
    if (unit0 >= G.syn_end) return;   // the warp's unit lies past the tile (uniform per warp)
    const uint8_t* wd = sb + 4 * SB;
    const uint32_t f = (uint32_t)lane & (LPCW - 1);
    uint32_t cur = 0;
    uint32_t c_key = 0, c_best = 0, c_tot = 0;   // the cell's reduction over its halves (HALVES == 2)
#pragma unroll 1
    for (uint32_t h = 0; h < HALVES; h++) {
        const uint32_t so = (uint32_t)wib * UNIT + h * 512u + (uint32_t)lane * 16;
        const uint32_t off = pos + so;
        const bool on = off < G.syn_end;
        uint32_t act0 = 0, en0 = 0;
        if (on) {
            if ((lane & (LPD - 1)) == 0) act0 = wd[(off >> SPD_L2) - ((pos >> SPD_L2) & ~15u)];
            // The cell's energy for the folded ssc_cycle, loaded before the
            // gathers so its latency overlaps them.
            if (!TUFT && A.ssc_soma && (lane & (LPD - 1)) == 0) en0 = A.cel_en[off >> SPD_L2];
            if (TUFT && h == 0) {
                const uint32_t ci = (off >> S_L2) - ((pos >> S_L2) & ~15u);
                if (LPC >= 8) {
                    if (f < 4) cur = wd[(1 + f) * WIN + ci];
                } else if (f == 0) {
                    cur = (uint32_t)wd[WIN + ci] | ((uint32_t)wd[2 * WIN + ci] << 8) |
                          ((uint32_t)wd[3 * WIN + ci] << 16) | ((uint32_t)wd[4 * WIN + ci] << 24);
                }
            }
        }
        uint32_t sum = 0, raw = 0;
        if (on) {
            const uint4 str4 = *(const uint4*)(sb + 2 * SB + so);
            const uint4 st4 = *(const uint4*)(sb + 3 * SB + so);
            const uint4 g0 = *(const uint4*)(sb + 2 * so);
            const uint4 g1 = *(const uint4*)(sb + 2 * so + 16);
            const uint32_t gw[8] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w};
            const uint32_t strw[4] = {str4.x, str4.y, str4.z, str4.w};
            const uint32_t stw[4] = {st4.x, st4.y, st4.z, st4.w};
            uint32_t nst[4], nfl[4];
#pragma unroll
            for (int w = 0; w < 4; w++) {
                const uint32_t lo = gw[2 * w], hi = gw[2 * w + 1];
                nst[w] = pack4(halo[lo & 0x7FFFu], halo[(lo >> 16) & 0x7FFFu], halo[hi & 0x7FFFu],
                               halo[(hi >> 16) & 0x7FFFu]);
            }
#pragma unroll
            for (int w = 0; w < 4; w++) {
                nfl[w] = nz_bits(stw[w]) >> 3;
                raw = __dp4a(nst[w], 0x01010101u, raw);
                sum = __dp4a(nst[w] & ~sign_bytes(strw[w]), 0x01010101u, sum);
            }
            *(uint4*)(A.st + off) = make_uint4(nst[0], nst[1], nst[2], nst[3]);
            *(uint4*)(A.fl + off) = make_uint4(nfl[0], nfl[1], nfl[2], nfl[3]);
        }
#pragma unroll
        for (uint32_t m = 1; m < LPD; m <<= 1) {
            sum += __shfl_xor_sync(0xFFFFFFFFu, sum, m);
            raw += __shfl_xor_sync(0xFFFFFFFFu, raw, m);
        }
        const bool lead = on && (lane & (LPD - 1)) == 0;
        const uint32_t den = off >> SPD_L2;
        uint32_t d_raw = 0, d_st = 0;
        if (lead) {
            const int active = sum > A.thresh;
            const uint32_t s2 = active ? sum : 0u;
            const uint32_t seed = (raw + A.thresh) | (den + A.den_idz);
            A.den_act[den] = update_activity((uint8_t)act0, active, rnd, (int32_t)seed, kDendriteActivityDecay);
            d_raw = min(raw >> 4, 255u);
            d_st = min(s2 >> 4, 255u);
            A.den_raw[den] = (uint8_t)d_raw;
            if (!TUFT && A.ssc_soma) d_st = ssc_soma(A.cel_en, den, en0, d_st);
            A.den_st[den] = (uint8_t)d_st;
        }
        if (!TUFT) continue;
        constexpr uint32_t kDenMask = (1u << (S_L2 - SPD_L2)) - 1;   // dendrite index within its cell
        uint32_t key = lead ? ((d_raw << 16) | (0xFFFFu - (den & kDenMask))) : 0u;
        uint32_t best = d_st, tot = d_st;
        if (HALVES == 2) {
            c_key = max(c_key, key);
            c_best = max(c_best, best);
            c_tot += tot;
            continue;
        }
        if (LPC == 32) {
            key = __reduce_max_sync(0xFFFFFFFFu, key);
            best = __reduce_max_sync(0xFFFFFFFFu, best);
            tot = __reduce_add_sync(0xFFFFFFFFu, tot);
        } else {
#pragma unroll
            for (uint32_t m = LPD; m < LPC; m <<= 1) {
                key = max(key, __shfl_xor_sync(0xFFFFFFFFu, key, m));
                best = max(best, __shfl_xor_sync(0xFFFFFFFFu, best, m));
                tot += __shfl_xor_sync(0xFFFFFFFFu, tot, m);
            }
            if (LPD > 1 && LPC >= 8) {
                const int src = lane & ~(int)(LPD - 1);
                key = __shfl_sync(0xFFFFFFFFu, key, src);
                best = __shfl_sync(0xFFFFFFFFu, best, src);
                tot = __shfl_sync(0xFFFFFFFFu, tot, src);
            }
        }
        c_key = key;
        c_best = best;
        c_tot = tot;
    }
    if (!TUFT) return;
    if (HALVES == 2) {
        c_key = __reduce_max_sync(0xFFFFFFFFu, c_key);
        c_best = __reduce_max_sync(0xFFFFFFFFu, c_best);
        c_tot = __reduce_add_sync(0xFFFFFFFFu, c_tot);
    }
    const uint32_t off = pos + (uint32_t)wib * UNIT + (uint32_t)lane * 16;   // in the cell's first half
    if (off < G.syn_end && (LPC >= 8 ? f < 8 : f == 0)) {
        const uint32_t c = off >> S_L2;
        const uint32_t best_raw = c_key >> 16;
        const uint32_t best_id = best_raw ? (0xFFFFu - (c_key & 0xFFFFu)) : 0u;
        const bool is_max = c_tot >= (1u << (A.mad_l2 + 8));
        const uint32_t tst = is_max ? 255u : ((c_tot >> A.mad_l2) & 0xFFu);
        if (LPC >= 8) {
            const uint32_t nv = f == 4 ? best_id : f == 5 ? best_raw : f == 6 ? c_best : tst;
            (&A.t_pid)[f][c] = (uint8_t)(f < 4 ? cur : nv);
        } else {
            A.t_pid[c] = (uint8_t)cur;
            A.t_praw[c] = (uint8_t)(cur >> 8);
            A.t_pst[c] = (uint8_t)(cur >> 16);
            A.t_ptft[c] = (uint8_t)(cur >> 24);
            A.t_bid[c] = (uint8_t)best_id;
            A.t_braw[c] = (uint8_t)best_raw;
            A.t_bst[c] = (uint8_t)c_best;
            A.t_st[c] = (uint8_t)tst;
        }
    }
}

// Raises the CTA's abort flag. The thread that raises it first records the
// give-up in the error bits of the area it was serving (its bounded wait ran
// out); the others' waits then end at once.
__device__ __forceinline__ void raise_abort(volatile int& s_abort, AreaCtl* ctl) {
    if (atomicExch((int*)&s_abort, 1) == 0 && ctl) atomicOr(&ctl->error, kErrWaitTimeout);
}

// The producer lane's ring position and fault-injection state.
struct ProducerState {
    uint32_t pb = 0, pround = 0;   // next buffer, and its round
    uint64_t issued = 0;           // stages issued (withheld ones included)
    uint64_t stall = 0;            // withhold the stage issued as number `stall` (counted from 1; 0: none)
    int withheld = -1;             // buffer of the withheld stage (-1: none)
    uint32_t limit_us = 0;         // bounded-wait limit
};

// Producer lane: issues every stage of tile G into the ring. False when a
// bounded wait gave up. A stage withheld for fault injection is neither
// copied nor armed, so its full barrier never completes and the consumers'
// bounded wait runs out; the producer cannot use that buffer again (its
// release never comes), so it is the buffer's last use.
template <bool TUFT, int MODE, bool FCLEAN>
__device__ __forceinline__ bool produce_tile(const FusedTuftArgs& A, const TileGeo& G, uint8_t* stages,
                                             uint64_t* full, uint64_t* empty, ProducerState& ps,
                                             volatile int& s_abort) {
    const uint32_t SB = stage_syns<MODE, FCLEAN>(A.stage_bytes);
    const uint32_t buf_bytes = A.stage_stride;
    const uint32_t nst = A.nst;
    for (uint32_t pos = G.syn0; pos < G.syn_end; pos += SB) {
        if (s_abort) return false;
        uint32_t& pb = ps.pb;
        // Buffer pb's previous use (round pround - 1) must be released.
        if (ps.pround > 0 && !mbar_wait(&empty[pb], (ps.pround - 1) & 1, ps.limit_us)) {
            raise_abort(s_abort, A.ctl);
            return false;
        }
        if (++ps.issued == ps.stall) {
            ps.withheld = (int)pb;
            if (++pb == nst) { pb = 0; ps.pround++; }
            continue;
        }
        const uint32_t left = G.syn_end - pos;
        const uint32_t nb = left < SB ? left : SB;
        uint8_t* dst = stages + (size_t)pb * buf_bytes;
        uint32_t n_arr_bytes = (MODE == 0 ? 2 * nb : 3 * nb) + nb + nb + (FCLEAN ? 0 : nb);
        // Windows of the stage's dendrites and cells, widened to 16-byte bounds.
        const uint32_t d0 = (pos >> A.spd_l2) & ~15u, d1 = (((pos + nb) >> A.spd_l2) + 15) & ~15u;
        const uint32_t c0 = (pos >> A.S_l2) & ~15u, c1 = (((pos + nb) >> A.S_l2) + 15) & ~15u;
        if (A.win) n_arr_bytes += (uint32_t)(d1 - d0) + (TUFT ? 4 * (uint32_t)(c1 - c0) : 0u);
        mbar_arrive_expect_tx(&full[pb], n_arr_bytes);
        if (A.win) {
            uint8_t* wd = dst + 4 * A.stage_bytes;
            bulk_g2s(wd, A.den_act + d0, (uint32_t)(d1 - d0), &full[pb]);
            if (TUFT) {
                const uint32_t cb = (uint32_t)(c1 - c0);
                bulk_g2s(wd + A.win_bytes, A.t_bid + c0, cb, &full[pb]);
                bulk_g2s(wd + 2 * A.win_bytes, A.t_braw + c0, cb, &full[pb]);
                bulk_g2s(wd + 3 * A.win_bytes, A.t_bst + c0, cb, &full[pb]);
                bulk_g2s(wd + 4 * A.win_bytes, A.t_st + c0, cb, &full[pb]);
            }
        }
        if (MODE == 0) {
            bulk_g2s(dst, A.gidx + pos, 2 * nb, &full[pb]);
        } else {
            bulk_g2s(dst, A.slc + pos, nb, &full[pb]);
            bulk_g2s(dst + SB, A.vofs + pos, nb, &full[pb]);
            bulk_g2s(dst + 2 * SB, A.uofs + pos, nb, &full[pb]);
        }
        bulk_g2s(dst + arr_off<MODE>(0, SB), A.str + pos, nb, &full[pb]);
        bulk_g2s(dst + arr_off<MODE>(1, SB), A.st + pos, nb, &full[pb]);
        if (!FCLEAN) bulk_g2s(dst + arr_off<MODE>(2, SB), A.fl + pos, nb, &full[pb]);
        if (++pb == nst) { pb = 0; ps.pround++; }
    }
    return true;
}

// After a give-up (or a withheld stage): let this CTA's copies land before
// its shared memory is released -- the latest armed use of every buffer must
// complete. A withheld stage was its buffer's last use and was never armed,
// so that buffer's latest armed use is the one before it.
__device__ __forceinline__ void producer_drain(uint64_t* full, uint32_t nst, const ProducerState& ps) {
    for (uint32_t b = 0; b < nst; b++) {
        uint64_t uses = ps.issued / nst + (b < ps.issued % nst ? 1 : 0);
        if ((int)b == ps.withheld) uses--;
        if (uses) mbar_wait(&full[b], (uint32_t)((uses - 1) & 1), ps.limit_us);
    }
}

// Consumer warps: take tile G's footprint -- load it as a tensor box and
// fire it in place, or stage it themselves -- then process the tile's stages
// from the ring (position `ring`). The caller's barrier before each
// tile (every consumer warp done with the previous footprint, its shared
// memory writes fenced for the async proxy) is what lets the box overwrite
// the footprint, so consumer thread 0 issues it right there: the footprint
// has one owner at a time whatever mix of tile forms a CTA takes. False when
// this warp gave up (a bounded wait ran out, or a give-up elsewhere was
// seen); the consumer warps then leave together at the next tile's barrier,
// whose OR-reduction keeps that decision uniform.
template <bool TUFT, int MODE, bool FCLEAN, int GEOM>
__device__ __forceinline__ bool consume_tile(const FusedTuftArgs& A, const TileGeo& G, uint8_t* halo, uint8_t* stages,
                                             uint64_t* full, uint64_t* empty, uint64_t* fp_full, uint32_t& ring,
                                             int lane, int wib, int32_t rnd, uint32_t limit_us,
                                             volatile int& s_abort) {
    if (A.fp_tma) {
        if (wib == 0 && lane == 0) {
            mbar_arrive_expect_tx(fp_full, A.fp_bytes);
            tma_load_3d(halo, &A.tmap, G.ulo - (int32_t)G.xoff, G.vlo, 0, fp_full);
        }
        const uint32_t fph = (ring & kFpPhase) ? 1u : 0u;
        bool got = !s_abort && mbar_wait(fp_full, fph, limit_us);
        got = __all_sync(0xFFFFFFFFu, got);
        if (!got && lane == 0) raise_abort(s_abort, A.ctl);
        if (consumers_sync_or(!got)) {
            // Let the box land before the CTA's shared memory is released.
            if (wib == 0 && lane == 0) mbar_wait(fp_full, fph, limit_us);
            ring ^= kFpPhase;
            return false;
        }
        ring ^= kFpPhase;
        fire_footprint(halo, A.fp_bytes);
        fence_proxy_async_smem();   // the next tile's load overwrites these bytes
    } else {
        build_footprint(A, G, halo, lane, wib);
        fence_proxy_async_smem();   // a later tile's box may overwrite these bytes
    }
    consumers_sync();
    const uint32_t SB = stage_syns<MODE, FCLEAN>(A.stage_bytes);
    const uint32_t cpu = A.chunks_per_unit;
    const uint32_t n_units_tile = cpu > 1 ? G.h * G.w : (G.syn_end - G.syn0 + 511) >> 9;
    for (uint32_t pos = G.syn0; pos < G.syn_end; pos += SB) {
        const uint32_t cb = ring & kRingBuf;
        bool got = !s_abort && mbar_wait(&full[cb], (ring & kRingPhase) ? 1u : 0u, limit_us);
        got = __all_sync(0xFFFFFFFFu, got);
        if (!got) {
            if (lane == 0) raise_abort(s_abort, A.ctl);
            return false;
        }
        if constexpr (GEOM == 0)
            tma_stage<TUFT, MODE, FCLEAN>(A, G, halo, stages + (size_t)cb * A.stage_stride, pos, n_units_tile, lane,
                                          wib, rnd);
        else
            stage_fast<TUFT, geom_spd_l2(GEOM), geom_lpc_l2(GEOM)>(A, G, halo, stages + (size_t)cb * A.stage_stride,
                                                                   pos, lane, wib, rnd);
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[cb]);
        ring = cb + 1 == A.nst ? (ring & ~kRingBuf) ^ kRingPhase : ring + 1;
    }
    return true;
}

// Shared-memory barriers of a CTA: the ring's full[nst] and empty[nst], then
// the footprint's at a fixed slot (nst <= 4).
constexpr uint32_t kFpFullSlot = 8;

template <bool TUFT, int MODE, bool FCLEAN, int GEOM>
__device__ __forceinline__ void tma_body(const FusedTuftArgs& A, uint8_t* smem, volatile int& s_abort) {
    uint64_t* full = (uint64_t*)(smem + A.ring_off);   // [nst]
    uint64_t* empty = full + A.nst;                    // [nst]
    uint64_t* fp_full = full + kFpFullSlot;
    uint8_t* stages = smem + A.ring_off + 128;
    uint8_t* halo = smem;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int wib = tid >> 5;
    const uint32_t limit_us = wait_limit_us(A.ctl);
    if (wib == kWarps) {
        // ---- producer: lane 0 streams every stage of this CTA's tiles ----
        if (lane != 0) return;
        ProducerState ps;
        ps.limit_us = limit_us;
        ps.stall = blockIdx.x == 0 ? A.ctl->stall_stage : 0u;
        for (uint32_t t = blockIdx.x; t < A.n_tiles && !s_abort; t += gridDim.x)
            if (!produce_tile<TUFT, MODE, FCLEAN>(A, tile_geo(A, t), stages, full, empty, ps, s_abort)) break;
        if (s_abort || ps.withheld >= 0) producer_drain(full, A.nst, ps);
        return;
    }
    // ---- consumer warps ----
    const int32_t rnd = rnd_at(A.rnd_key, cycle_of(A));
    uint32_t ring = 0;
    bool ok = true;
    for (uint32_t t = blockIdx.x; t < A.n_tiles; t += gridDim.x) {
        const TileGeo G = tile_geo(A, t);
        // Every consumer is done with the previous tile; all leave together
        // if any gave up.
        if (consumers_sync_or(!ok || s_abort)) break;
        ok = consume_tile<TUFT, MODE, FCLEAN, GEOM>(A, G, halo, stages, full, empty, fp_full, ring, lane, wib, rnd,
                                                    limit_us, s_abort);
    }
}

__device__ __forceinline__ void init_ring(uint8_t* ring, uint32_t nst, volatile int& s_abort) {
    uint64_t* full = (uint64_t*)ring;
    uint64_t* empty = full + nst;
    if (threadIdx.x == 0) {
        for (uint32_t i = 0; i < nst; i++) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], kWarps);
        }
        mbar_init(full + kFpFullSlot, 1);
        fence_mbar_init();
        s_abort = 0;
    }
    __syncthreads();
}

// Gather form (bit 1: sources outside the footprint) and flags state (bit 0:
// foreign flag bits) of a tuft, from its verification status.
__device__ __forceinline__ uint32_t mode_of(const FusedTuftArgs& A) {
    const uint32_t status = A.ctl->tuft_status[A.status_idx];
    return ((status & kTuftSrcOutsideTile) ? 2u : 0u) | ((status & kTuftFlagsForeign) ? 1u : 0u);
}

template <bool TUFT>
__global__ void __launch_bounds__(kThreads, 3) k_fused_tuft_tma(const __grid_constant__ FusedTuftArgs A) {
    pdl_begin();
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ volatile int s_abort;   // a bounded wait gave up
    init_ring(smem + A.ring_off, A.nst, s_abort);
    // One specialised body per gather mode and flags state (uniform per launch).
    switch (mode_of(A)) {
    case 0:
        // Shapes with a specialised consumer (pyramidal tufts, or the
        // one-dendrite cells of spiny stellates).
        if (TUFT) {
            switch (A.geom) {
            case 3: tma_body<TUFT, 0, true, 3>(A, smem, s_abort); return;
            case 4: tma_body<TUFT, 0, true, 4>(A, smem, s_abort); return;
            case 5: tma_body<TUFT, 0, true, 5>(A, smem, s_abort); return;
            case 6: tma_body<TUFT, 0, true, 6>(A, smem, s_abort); return;
            case 7: tma_body<TUFT, 0, true, 7>(A, smem, s_abort); return;
            case 8: tma_body<TUFT, 0, true, 8>(A, smem, s_abort); return;
            default: break;
            }
        } else {
            switch (A.geom) {
            case 1: tma_body<TUFT, 0, true, 1>(A, smem, s_abort); return;
            case 2: tma_body<TUFT, 0, true, 2>(A, smem, s_abort); return;
            default: break;
            }
        }
        tma_body<TUFT, 0, true, 0>(A, smem, s_abort);
        break;
    case 1: tma_body<TUFT, 0, false, 0>(A, smem, s_abort); break;
    case 2: tma_body<TUFT, 1, true, 0>(A, smem, s_abort); break;
    default: tma_body<TUFT, 1, false, 0>(A, smem, s_abort); break;
    }
}

// ------------------------------------------------------- batched form ----
// One launch over the tiles of several tufts (the same tuft step of several
// areas): job j owns global tiles tile0[j] .. tile0[j + 1] - 1. Persistent
// CTAs walk the global tiles in the same stride as the one-tuft kernel. The
// job table is the launch's own parameter block (__grid_constant__): it is
// read-only there, so the compiler keeps argument fields in registers across
// the stores of a stage, and nothing needs copying per job. Every job of a
// launch shares the ring geometry (nst, stage_stride, ring_off).
// As many argument blocks as fit the 32 KB kernel parameter limit.
constexpr uint32_t kMaxBatchJobs = (32764 - 16) / (sizeof(FusedTuftArgs) + 4) - 1;

struct BatchParams {
    FusedTuftArgs jobs[kMaxBatchJobs];
    uint32_t tile0[kMaxBatchJobs + 1];
    uint32_t n_jobs, nst, ring_off;
};
static_assert(sizeof(BatchParams) <= 32764, "batched tuft parameter block exceeds the kernel parameter limit");

// The job of global tile t: tile0[j] <= t < tile0[j + 1].
__device__ __forceinline__ uint32_t job_of(const BatchParams& P, uint32_t t) {
    uint32_t lo = 0, hi = P.n_jobs;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (P.tile0[mid] <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <bool TUFT>
__global__ void __launch_bounds__(kThreads, 3) k_fused_tuft_batch(const __grid_constant__ BatchParams P) {
    pdl_begin();
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ volatile int s_abort;
    const uint32_t nst = P.nst;
    init_ring(smem + P.ring_off, nst, s_abort);
    uint64_t* full = (uint64_t*)(smem + P.ring_off);
    uint64_t* empty = full + nst;
    uint64_t* fp_full = full + kFpFullSlot;
    uint8_t* stages = smem + P.ring_off + 128;
    uint8_t* halo = smem;
    const uint32_t n_tiles = P.tile0[P.n_jobs];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int wib = tid >> 5;
    if (wib == kWarps) {
        if (lane != 0) return;
        uint32_t cur = 0xFFFFFFFFu, mode = 0;
        ProducerState ps;
        AreaCtl* ctl = nullptr;
        for (uint32_t t = blockIdx.x; t < n_tiles && !s_abort; t += gridDim.x) {
            const uint32_t j = job_of(P, t);
            const FusedTuftArgs& A = P.jobs[j];
            if (j != cur) {
                cur = j;
                mode = mode_of(A);
                ctl = A.ctl;
                // Waits follow the job's area. The fault hook: the CTA that
                // takes a job's first tile withholds the job area's
                // stall_stage-th stage from that tile on.
                ps.limit_us = wait_limit_us(ctl);
                if (t == P.tile0[j] && ctl->stall_stage) ps.stall = ps.issued + ctl->stall_stage;
            }
            const TileGeo G = tile_geo(A, t - P.tile0[j]);
            bool ok;
            switch (mode) {
            case 0: ok = produce_tile<TUFT, 0, true>(A, G, stages, full, empty, ps, s_abort); break;
            case 1: ok = produce_tile<TUFT, 0, false>(A, G, stages, full, empty, ps, s_abort); break;
            case 2: ok = produce_tile<TUFT, 1, true>(A, G, stages, full, empty, ps, s_abort); break;
            default: ok = produce_tile<TUFT, 1, false>(A, G, stages, full, empty, ps, s_abort); break;
            }
            if (!ok) break;
        }
        if (s_abort || ps.withheld >= 0) producer_drain(full, nst, ps);
        return;
    }
    uint32_t cur = 0xFFFFFFFFu, mode = 0, ring = 0;
    int32_t rnd = 0;
    uint32_t limit_us = 0;
    bool ok = true;
    for (uint32_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const uint32_t j = job_of(P, t);
        const FusedTuftArgs& A = P.jobs[j];
        // Every consumer is done with the previous tile; all leave together
        // if any gave up.
        if (consumers_sync_or(!ok || s_abort)) break;
        if (j != cur) {
            cur = j;
            mode = mode_of(A);
            rnd = rnd_at(A.rnd_key, cycle_of(A));
            limit_us = wait_limit_us(A.ctl);
        }
        const TileGeo G = tile_geo(A, t - P.tile0[j]);
#define BM_CONSUME(M, FC, GM)                                                                                   \
    ok = consume_tile<TUFT, M, FC, GM>(A, G, halo, stages, full, empty, fp_full, ring, lane, wib, rnd, limit_us, \
                                       s_abort)
        switch (mode) {
        case 0:
            if (TUFT) {
                switch (A.geom) {
                case 3: BM_CONSUME(0, true, 3); break;
                case 4: BM_CONSUME(0, true, 4); break;
                case 5: BM_CONSUME(0, true, 5); break;
                case 6: BM_CONSUME(0, true, 6); break;
                case 7: BM_CONSUME(0, true, 7); break;
                case 8: BM_CONSUME(0, true, 8); break;
                default: BM_CONSUME(0, true, 0); break;
                }
            } else {
                switch (A.geom) {
                case 1: BM_CONSUME(0, true, 1); break;
                case 2: BM_CONSUME(0, true, 2); break;
                default: BM_CONSUME(0, true, 0); break;
                }
            }
            break;
        case 1: BM_CONSUME(0, false, 0); break;
        case 2: BM_CONSUME(1, true, 0); break;
        default: BM_CONSUME(1, false, 0); break;
        }
#undef BM_CONSUME
    }
}

// ------------------------------------------------------ source compile ----
// Writes each synapse's gather offset into its tile's footprint
// (gather_offset) and sets kTuftSrcOutsideTile if a source cannot be served
// from the footprint, kTuftFlagsForeign if a flag byte has bits other than
// SYN_PREV_ACTIVE. 16 synapses (of one cell) per thread. With gidx == nullptr
// (untiled tufts) only the flags are checked.
__global__ void k_compile_tuft(const uint8_t* __restrict__ slc, const int8_t* __restrict__ vo,
                               const int8_t* __restrict__ uo, const uint8_t* __restrict__ fl, uint16_t* gidx,
                               uint64_t n, GatherGeo g, unsigned int* status) {
    pdl_begin();
    uint32_t bits = 0;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * 16; i < n;
         i += (uint64_t)gridDim.x * blockDim.x * 16) {
        const uint4 f4 = *(const uint4*)(fl + i);
        const uint32_t* fw4 = (const uint32_t*)&f4;
#pragma unroll
        for (int w = 0; w < 4; w++)
            if (fw4[w] & 0xEFEFEFEFu) bits |= kTuftFlagsForeign;
        if (!gidx) continue;
        const uint4 s4 = *(const uint4*)(slc + i), v4 = *(const uint4*)(vo + i), u4 = *(const uint4*)(uo + i);
        const uint32_t* sw = (const uint32_t*)&s4;
        const uint32_t* vw = (const uint32_t*)&v4;
        const uint32_t* uw = (const uint32_t*)&u4;
        uint32_t out[8];
#pragma unroll
        for (int w = 0; w < 4; w++) {
            uint32_t o[4];
#pragma unroll
            for (int b = 0; b < 4; b++) {
                bool ok;
                o[b] = gather_offset(g, i, (sw[w] >> (8 * b)) & 0xFF, (int)(int8_t)(vw[w] >> (8 * b)),
                                     (int)(int8_t)(uw[w] >> (8 * b)), ok);
                if (!ok) bits |= kTuftSrcOutsideTile;
            }
            out[2 * w] = o[0] | (o[1] << 16);
            out[2 * w + 1] = o[2] | (o[3] << 16);
        }
        uint4* dst = (uint4*)(gidx + i);
        dst[0] = make_uint4(out[0], out[1], out[2], out[3]);
        dst[1] = make_uint4(out[4], out[5], out[6], out[7]);
    }
    bits = __reduce_or_sync(0xFFFFFFFFu, bits);
    if ((threadIdx.x & 31) == 0 && bits) atomicOr(status, bits);
}

inline int ilog2(uint64_t x) {
    int l = 0;
    while ((1ull << l) < x) l++;
    return l;
}
inline bool pow2(uint64_t x) { return x && !(x & (x - 1)); }

}  // namespace

namespace {

// Stages of the shared-memory ring: the deepest ring of at most max_n stages
// with which three CTAs share an SM, else with which two do. Measured on
// B200: one tuft alone (area_256, 64K-synapse tiles) runs fastest with three
// stages (four no longer leave room for three CTAs per SM), batched steps
// (many tufts of several areas per launch) with up to four.
uint32_t ring_stages(uint64_t stride, uint64_t halo, uint32_t max_n) {
    for (uint32_t n = max_n; n >= 2; n--)
        if (128 + n * stride + halo <= kSmem3) return n;
    for (uint32_t n = max_n; n >= 2; n--)
        if (128 + n * stride + halo <= kMaxSmem) return n;
    return 2;
}

// Largest default tile, in synapses (an explicit target may ask for more).
constexpr uint64_t kMaxTileSyns = 65536;

int device_sms() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
    return sms;
}

// Launch parameters of tuft t of data layer i (gidx left null). `target` is
// the synapses per tile to aim for (0: chosen from the tuft's size);
// `allow_tma` lets the footprint come from a tensor box load.
void plan_tuft(FusedTuft& FT, const bm_area_plan& P, uint32_t i, uint32_t t, int sms, uint32_t target_syns = 0,
               bool allow_tma = true) {
    const bm_layer_plan& L = P.layers[i];
    bool aligned = true;
    for (int k = 0; k < BM_BUF_COUNT; k++)
        if (L.buf_off[k] != UINT64_MAX && (L.buf_off[k] % 16)) aligned = false;
    const bm_tuft_plan& T = L.tufts[t];
    FT = FusedTuft{};
    uint32_t spd = T.syns_per_den, dpt = T.dens_per_tft;
    FT.ok = aligned && pow2(spd) && spd >= 16 && spd <= 512 && pow2(dpt) && (T.syn_idz % 16) == 0;
    // Fast gathers serve the pool's distinct slices when their ids are
    // contiguous and spatial (mid 0, where bismit's scalar and vec4 index
    // forms agree); anything else takes the general per-synapse path.
    uint32_t lo = 255, hi = 0;
    for (uint32_t k = 0; k < T.n_src_uniq; k++) {
        lo = std::min<uint32_t>(lo, T.src_uniq_slc_ids[k]);
        hi = std::max<uint32_t>(hi, T.src_uniq_slc_ids[k]);
    }
    uint32_t nrec = (T.n_src_uniq && hi - lo + 1 <= (uint32_t)kMaxRecs) ? hi - lo + 1 : 0;
    for (uint32_t k = 0; k < nrec; k++)
        if (P.slc_v_mid[lo + k] || P.slc_u_mid[lo + k] || !P.slc_v_scale[lo + k]) nrec = 0;
    FT.slc0 = nrec ? lo : 0;
    FT.nrec = nrec;
    if (!FT.ok) return;
    // Tiled gathers: the recorded slices share one geometry; the
    // footprint margin is the pool's largest offset.
    bool same = nrec > 0;
    for (uint32_t k = 1; k < nrec && same; k++) {
        uint32_t a = lo, b = lo + k;
        same = P.slc_v_size[a] == P.slc_v_size[b] && P.slc_u_size[a] == P.slc_u_size[b] &&
               P.slc_v_scale[a] == P.slc_v_scale[b] && P.slc_u_scale[a] == P.slc_u_scale[b];
    }
    int rv = 0, ru = 0;
    for (uint32_t k = 0; k < T.n_src_uniq && same; k++) {
        int a, b;
        uint8_t sid = T.src_uniq_slc_ids[k];
        if (!offset_extent(T.src_uniq_reaches[k], P.slc_v_scale[sid], P.slc_u_scale[sid], &a, &b)) same = false;
        rv = std::max(rv, a);
        ru = std::max(ru, b);
    }
    if (!same) return;
    const uint32_t S = T.syns_per_tft;
    const uint32_t cpu = S > 512 ? S / 512 : 1;
    const uint32_t SB = kWarps * cpu * 512;
    const uint64_t n_syn = (uint64_t)L.cells * S;
    uint64_t target = std::min<uint64_t>(kMaxTileSyns, std::max<uint64_t>(4096, n_syn / ((uint64_t)sms * 16)));
    if (target_syns) target = target_syns;
    const uint64_t cells = std::max<uint64_t>(1, target / S);
    const uint32_t vs = P.slc_v_scale[lo], us = P.slc_u_scale[lo];
    // Tiles are whole rows (H of them) when `cells` covers a row, else a row
    // cut into k equal parts, k the nearest whole number of `cells`-wide
    // parts (no sliver at the row's end). The tile narrows until its
    // footprint fits the 16-bit gather offsets.
    uint32_t W, H, k = 1;
    if (cells >= L.u_size) {
        W = L.u_size;
        H = (uint32_t)std::min<uint64_t>(L.v_size, cells / L.u_size);
    } else {
        k = (uint32_t)std::max<uint64_t>(1, (L.u_size + cells / 2) / cells);
        W = (L.u_size + k - 1) / k;
        H = 1;
    }
    uint64_t frows, fw, fsz, halo;
    for (;;) {
        frows = ((uint64_t)(H - 1) * vs + 15) / 16 + 1 + 2 * (uint64_t)rv;
        fw = ((uint64_t)(W - 1) * us + 15) / 16 + 1 + 2 * (uint64_t)ru;
        fsz = frows * fw;
        halo = (uint64_t)nrec * fsz;
        if (halo < 32768) break;
        if (H > 1) {
            H--;
        } else if (W > 1) {
            k++;
            W = (L.u_size + k - 1) / k;
        } else {
            return;   // even one cell's footprint is too large for 16-bit offsets
        }
    }
    // The footprint by tensor box: a 3-D view (column, row, slice) of the
    // recorded slices, which must lie back to back with rows of a multiple of
    // 16 bytes. A box starts on a 16-byte column boundary, so its rows are
    // up to 15 bytes wider than the footprint's.
    bool tma = allow_tma && P.slc_u_size[lo] % 16 == 0 && P.slc_axn_idz[lo] % 16 == 0;
    for (uint32_t k = 1; k < nrec && tma; k++)
        tma = P.slc_axn_idz[lo + k] == P.slc_axn_idz[lo] + k * P.slc_v_size[lo] * P.slc_u_size[lo];
    // Row pitch and shared-memory banks: a warp's byte gathers reach up to
    // 2 * rv + 1 rows of one cell's neighbourhood, and rows whose pitch puts
    // the same column in the same bank cost a wavefront each. A pitch of an
    // odd number of words spreads 32 consecutive rows over every bank; a box
    // row (a multiple of 16 bytes) does best at 16 bytes past a multiple of
    // 32 (8 rows before a bank repeats, against 4 or fewer otherwise).
    uint64_t fwb = (fw + 15 + 15) / 16 * 16;
    if (fwb % 32 == 0 && fwb + 16 <= 256 && (uint64_t)nrec * frows * (fwb + 16) < 32768) fwb += 16;
    tma = tma && fwb <= 256 && frows <= 256 && (uint64_t)nrec * frows * fwb < 32768;
    if (tma) {
        fw = fwb;
    } else {
        const uint64_t fwo = fw + (12 - fw % 8) % 8;   // fw % 8 == 4: rows an odd number of words apart
        if ((uint64_t)nrec * frows * fwo < 32768) fw = fwo;
    }
    fsz = frows * fw;
    halo = (uint64_t)nrec * fsz;
    // Windows: up to SB / 16 dendrites (or cells) per stage, widened by 16
    // at both ends.
    const uint32_t win_bytes = SB / 16 + 32;
    const uint32_t buf_bytes = 4 * SB + 5 * win_bytes;
    // The footprint sits at the start of dynamic shared memory (gathers then
    // address it with a constant base), the ring after it.
    const uint64_t ring_off = ((halo + 127) / 128) * 128;
    const uint32_t nst = ring_stages(buf_bytes, ring_off, 3);
    // Gathers mask offsets to 15 bits: at least 32 KB of shared memory keeps
    // every masked offset inside the CTA's allocation.
    const uint64_t smem = std::max<uint64_t>(32768, ring_off + 128 + (uint64_t)nst * buf_bytes);
    if (smem > kMaxSmem) return;
    FT.tiled = true;
    FT.fp_tma = tma;
    FT.tile_w = W;
    FT.tile_h = H;
    FT.rv = rv;
    FT.ru = ru;
    FT.fw = (uint32_t)fw;
    FT.frows = (uint32_t)frows;
    FT.fsz = (uint32_t)fsz;
    FT.nst = nst;
    FT.stage_bytes = SB;
    FT.stage_stride = buf_bytes;
    FT.win_bytes = win_bytes;
    FT.win = (T.den_idz % 16) == 0 && (T.cel_idz % 16) == 0;
    FT.ring_off = (uint32_t)ring_off;
    FT.smem = (uint32_t)smem;
    FT.src_vs = vs;
    FT.src_us = us;
    FT.src_vsz = P.slc_v_size[lo];
    FT.src_usz = P.slc_u_size[lo];
    for (uint32_t k = 0; k < nrec; k++) FT.src_idz[k] = P.slc_axn_idz[lo + k];
    // Persistent grid: as many CTAs as fit on the device at once.
    const bool pyr = L.kind == BM_LYR_PYRAMIDAL;
    auto kern = pyr ? k_fused_tuft_tma<true> : k_fused_tuft_tma<false>;
    // The cap is a property of the kernel, shared by every area on the device:
    // set it to the largest footprint any tuft may plan, never lower.
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, FT.smem) != cudaSuccess)
        per_sm = 1;
    const uint64_t n_tiles = (uint64_t)L.depth * ((L.u_size + W - 1) / W) * ((L.v_size + H - 1) / H);
    FT.grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(n_tiles, (uint64_t)sms * std::max(per_sm, 1)));
}

}  // namespace

int plan_fused(FusedArea& F, const bm_area_plan& P) {
    F.sms = device_sms();
    for (uint32_t i = 0; i < P.n_layers; i++)
        for (uint32_t t = 0; t < P.layers[i].n_tufts; t++) plan_tuft(F.t[i][t], P, i, t, F.sms);
    cudaGetLastError();
    return BM_OK;
}

int plan_fused_tuft(FusedArea& F, const bm_area_plan& P, uint32_t layer, uint32_t t) {
    F.sms = device_sms();
    plan_tuft(F.t[layer][t], P, layer, t, F.sms);
    cudaGetLastError();
    return BM_OK;
}

bool retile_fused_tuft(FusedArea& F, const bm_area_plan& P, uint32_t layer, uint32_t t, uint32_t target_syns,
                       bool* changed, bool staged) {
    *changed = false;
    FusedTuft& FT = F.t[layer][t];
    if (!FT.tiled || !FT.gidx) return false;
    FusedTuft next;
    plan_tuft(next, P, layer, t, F.sms, target_syns, !staged);
    cudaGetLastError();
    if (!next.tiled) return false;
    if (next.tile_w == FT.tile_w && next.tile_h == FT.tile_h && next.nst == FT.nst && next.smem == FT.smem &&
        next.fp_tma == FT.fp_tma) {
        FT.tile_target = target_syns;   // same tiles: the compiled offsets stay valid
        FT.fp_staged = staged;
        return true;
    }
    *changed = true;
    next.gidx = FT.gidx;
    next.tile_target = target_syns;
    next.fp_staged = staged;
    next.bound_axns = FT.bound_axns;
    FT = next;
    if (FT.bound_axns) bind_fused_tuft(F, P, layer, t, FT.bound_axns);
    return true;
}

int prepare_fused(FusedArea& F, const bm_area_plan& P, std::string* err) {
    int rc = plan_fused(F, P);
    if (rc != BM_OK) return rc;
    // Compiled gather offsets: 2 bytes per synapse of every tiled tuft.
    for (uint32_t i = 0; i < P.n_layers; i++)
        for (uint32_t t = 0; t < P.layers[i].n_tufts; t++) {
            FusedTuft& FT = F.t[i][t];
            if (!FT.tiled) continue;
            const uint64_t n_syn = (uint64_t)P.layers[i].cells * P.layers[i].tufts[t].syns_per_tft;
            const cudaError_t e = F.pool ? cudaMallocFromPoolAsync((void**)&FT.gidx, n_syn * sizeof(int16_t), F.pool,
                                                                   F.pool_stream)
                                         : cudaMalloc(&FT.gidx, n_syn * sizeof(int16_t));
            if (e != cudaSuccess) {
                cudaGetLastError();
                FT.gidx = nullptr;
                if (err) *err = "cudaMalloc of the gather offsets failed";
                free_fused(F, F.pool_stream);
                return BM_ERR_OOM;
            }
        }
    return BM_OK;
}

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled, resolved once through the runtime (the library does
// not link the driver library).
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        cudaGetLastError();
        return (EncodeTiledFn)p;
    }();
    return fn;
}

// The footprint box of tiled tuft FT over the axon space at `axns`: u8
// elements, dims (u_size, v_size, nrec) of the recorded slices, box (fw,
// frows, nrec); coordinates outside the slices read as 0.
bool encode_footprint_map(FusedTuft& FT, const bm_area_plan& P, const uint8_t* axns) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    const uint32_t lo = FT.slc0;
    const cuuint64_t dims[3] = {P.slc_u_size[lo], P.slc_v_size[lo], FT.nrec};
    const cuuint64_t strides[2] = {P.slc_u_size[lo], (cuuint64_t)P.slc_u_size[lo] * P.slc_v_size[lo]};
    const cuuint32_t box[3] = {FT.fw, FT.frows, FT.nrec};
    const cuuint32_t elem[3] = {1, 1, 1};
    CUtensorMap m;
    const CUresult r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, (void*)(axns + P.slc_axn_idz[lo]), dims, strides, box,
                           elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    static_assert(sizeof m == sizeof FT.tmap, "tensor map size");
    std::memcpy(FT.tmap, &m, sizeof m);
    return true;
}

}  // namespace

int bind_fused_tuft(FusedArea& F, const bm_area_plan& P, uint32_t layer, uint32_t t, const uint8_t* axns) {
    FusedTuft& FT = F.t[layer][t];
    FT.bound_axns = axns;
    if (!FT.tiled || !FT.fp_tma) return BM_OK;
    if (((uintptr_t)(axns + P.slc_axn_idz[FT.slc0]) & 15) == 0 && encode_footprint_map(FT, P, axns)) return BM_OK;
    // The driver refused the box: the consumers stage the footprint instead
    // (same tiles, rows without the column alignment).
    FusedTuft next;
    plan_tuft(next, P, layer, t, F.sms, FT.tile_target, false);
    cudaGetLastError();
    next.gidx = FT.gidx;
    next.tile_target = FT.tile_target;
    next.tile_tuned = FT.tile_tuned;
    next.fp_staged = FT.fp_staged;
    next.bound_axns = axns;
    FT = next;
    return BM_OK;
}

int bind_fused(FusedArea& F, const bm_area_plan& P, const uint8_t* axns) {
    for (uint32_t i = 0; i < P.n_layers; i++)
        for (uint32_t t = 0; t < P.layers[i].n_tufts; t++) bind_fused_tuft(F, P, i, t, axns);
    return BM_OK;
}

void free_fused(FusedArea& F, cudaStream_t s) {
    for (auto& row : F.t)
        for (auto& FT : row)
            if (FT.gidx) {
                if (F.pool) cudaFreeAsync(FT.gidx, s);
                else cudaFree(FT.gidx);
                FT.gidx = nullptr;
            }
}

namespace {

GatherGeo geo_of(const FusedTuft& FT, const DevLayer& L, const DevTuft& T) {
    GatherGeo g{};
    g.S_l2 = (uint32_t)ilog2(T.spt);
    g.cols = L.v_size * L.u_size;
    g.u_size = L.u_size;
    g.tile_w = FT.tiled ? FT.tile_w : 1;
    g.tile_h = FT.tiled ? FT.tile_h : 1;
    g.vs = FT.src_vs;
    g.us = FT.src_us;
    g.rv = FT.rv;
    g.ru = FT.ru;
    g.fw = FT.fw;
    g.fsz = FT.fsz;
    g.slc0 = FT.slc0;
    g.nrec = FT.nrec;
    g.xalign = FT.tiled && FT.fp_tma ? 1u : 0u;
    return g;
}

}  // namespace

GatherGeo gather_geo(const FusedArea& F, const bm_area_plan& P, uint32_t layer, uint32_t t) {
    DevLayer D;
    fill_dev_layer(D, P, layer, nullptr);
    return geo_of(F.t[layer][t], D, D.tft[t]);
}

void launch_compile_tuft(const FusedArea& F, const DevLayer& L, uint32_t layer, uint32_t t, AreaCtl* ctl,
                         cudaStream_t s) {
    const FusedTuft& FT = F.t[layer][t];
    if (!FT.ok) return;
    const DevTuft& T = L.tft[t];
    unsigned int* status = &ctl->tuft_status[layer * BM_MAX_TUFTS + t];
    cudaMemsetAsync(status, 0, sizeof(unsigned int), s);
    const uint64_t n = (uint64_t)L.cells * T.spt;
    const uint64_t threads = (n + 15) / 16;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((threads + 255) / 256, (uint64_t)F.sms * 8));
    launch_pdl(k_compile_tuft, grid, 256, 0, s, L.buf[BM_BUF_SYN_SRC_SLC_IDS] + T.syn_idz,
                                        (const int8_t*)L.buf[BM_BUF_SYN_SRC_COL_V_OFFS] + T.syn_idz,
                                        (const int8_t*)L.buf[BM_BUF_SYN_SRC_COL_U_OFFS] + T.syn_idz,
                                        L.buf[BM_BUF_SYN_FLAG_SETS] + T.syn_idz, FT.tiled ? FT.gidx : nullptr, n,
                                        geo_of(FT, L, T), status);
}

void launch_verify_tufts(const FusedArea& F, const DevLayer& L, uint32_t layer, AreaCtl* ctl, cudaStream_t s) {
    for (uint32_t t = 0; t < L.n_tufts; t++) launch_compile_tuft(F, L, layer, t, ctl, s);
}

namespace {

// The kernel arguments of tuft t of data layer `layer` (with ssc_cycle folded
// in when `ssc_soma`).
void make_args(FusedTuftArgs& A, const FusedArea& F, const uint8_t* axns, const SliceRec* slices, const DevLayer& L,
               uint32_t layer, uint32_t t, AreaCtl* ctl, bool ssc_soma) {
    const DevTuft& T = L.tft[t];
    const FusedTuft& FT = F.t[layer][t];
    std::memset(&A, 0, sizeof A);
    A.axns = axns;
    A.slices = slices;
    A.ctl = ctl;
    A.slc = L.buf[BM_BUF_SYN_SRC_SLC_IDS] + T.syn_idz;
    A.vofs = (const int8_t*)L.buf[BM_BUF_SYN_SRC_COL_V_OFFS] + T.syn_idz;
    A.uofs = (const int8_t*)L.buf[BM_BUF_SYN_SRC_COL_U_OFFS] + T.syn_idz;
    A.str = (const int8_t*)L.buf[BM_BUF_SYN_STRENGTHS] + T.syn_idz;
    A.st = L.buf[BM_BUF_SYN_STATES] + T.syn_idz;
    A.fl = L.buf[BM_BUF_SYN_FLAG_SETS] + T.syn_idz;
    A.gidx = FT.gidx;
    A.den_act = L.buf[BM_BUF_DEN_ACTIVITIES] + T.den_idz;
    A.den_raw = L.buf[BM_BUF_DEN_STATES_RAW] + T.den_idz;
    A.den_st = L.buf[BM_BUF_DEN_STATES] + T.den_idz;
    A.cel_en = L.buf[BM_BUF_CEL_ENERGIES];
    A.ssc_soma = ssc_soma && L.kind == BM_LYR_SPINY_STELLATE && T.dpt == 1 && T.den_idz == 0;
    const bool tuft = L.kind == BM_LYR_PYRAMIDAL;
    if (tuft) {
        A.t_pid = L.buf[BM_BUF_TFT_PREV_BEST_DEN_IDS] + T.cel_idz;
        A.t_praw = L.buf[BM_BUF_TFT_PREV_BEST_DEN_STATES_RAW] + T.cel_idz;
        A.t_pst = L.buf[BM_BUF_TFT_PREV_BEST_DEN_STATES] + T.cel_idz;
        A.t_ptft = L.buf[BM_BUF_TFT_PREV_STATES] + T.cel_idz;
        A.t_bid = L.buf[BM_BUF_TFT_BEST_DEN_IDS] + T.cel_idz;
        A.t_braw = L.buf[BM_BUF_TFT_BEST_DEN_STATES_RAW] + T.cel_idz;
        A.t_bst = L.buf[BM_BUF_TFT_BEST_DEN_STATES] + T.cel_idz;
        A.t_st = L.buf[BM_BUF_TFT_STATES] + T.cel_idz;
    }
    const uint64_t S = (uint64_t)T.spt;
    A.n_syn = (uint64_t)L.cells * S;
    A.den_idz = (uint32_t)T.den_idz;
    A.thresh = T.thresh;
    A.cols = L.v_size * L.u_size;
    A.u_size = L.u_size;
    A.v_size = L.v_size;
    A.S_l2 = ilog2(S);
    A.spd_l2 = ilog2(T.spd);
    A.lpd_l2 = A.spd_l2 - 4;
    A.lpc_l2 = std::min<uint32_t>(A.S_l2 - 4, 5);
    A.chunks_per_unit = S > 512 ? (uint32_t)(S / 512) : 1u;
    A.mad_l2 = T.mad_l2;
    A.slc0 = FT.slc0;
    A.nrec = FT.nrec;
    A.vec4 = (T.spt & 3) == 0;
    A.rnd_key = T.rnd_key_den;
    A.status_idx = layer * BM_MAX_TUFTS + t;
    if (FT.tiled) {
        A.tile_w = FT.tile_w;
        A.tile_h = FT.tile_h;
        A.tiles_u = (L.u_size + FT.tile_w - 1) / FT.tile_w;
        A.tiles_v = (L.v_size + FT.tile_h - 1) / FT.tile_h;
        A.n_tiles = L.depth * A.tiles_u * A.tiles_v;
        A.usz_magic = div_magic(L.u_size);
        A.per_slice_magic = div_magic(A.tiles_u * A.tiles_v);
        A.tiles_u_magic = div_magic(A.tiles_u);
        A.rv = FT.rv;
        A.ru = FT.ru;
        A.fw = FT.fw;
        A.frows = FT.frows;
        A.fsz = FT.fsz;
        A.src_vs = FT.src_vs;
        A.src_us = FT.src_us;
        A.src_vsz = FT.src_vsz;
        A.src_usz = FT.src_usz;
        for (uint32_t k = 0; k < FT.nrec; k++) A.src_idz[k] = FT.src_idz[k];
        A.nst = FT.nst;
        A.stage_bytes = FT.stage_bytes;
        A.ring_off = FT.ring_off;
        A.unit_l2 = 9 + ilog2(A.chunks_per_unit);
        A.stage_stride = FT.stage_stride;
        A.win = FT.win;
        A.win_bytes = FT.win_bytes;
        A.fp_tma = FT.fp_tma ? 1u : 0u;
        A.fp_bytes = FT.nrec * FT.fsz;
        if (FT.fp_tma) std::memcpy(&A.tmap, FT.tmap, sizeof A.tmap);
        A.geom = consumer_shape(FT, (uint32_t)S, T.spd, tuft);
    } else {
        A.n_units = S > 512 ? (uint64_t)L.cells : (A.n_syn + 511) / 512;
    }
}

}  // namespace

void launch_fused_tuft(const FusedArea& F, const uint8_t* axns, const SliceRec* slices, const DevLayer& L,
                       uint32_t layer, uint32_t t, AreaCtl* ctl, cudaStream_t s, bool ssc_soma, int64_t host_cycle) {
    const FusedTuft& FT = F.t[layer][t];
    FusedTuftArgs A;
    make_args(A, F, axns, slices, L, layer, t, ctl, ssc_soma);
    if (host_cycle >= 0) {
        A.cycle_from_host = 1;
        A.cycle = (unsigned long long)host_cycle;
    }
    const bool tuft = L.kind == BM_LYR_PYRAMIDAL;
    if (FT.tiled) {
        auto kern = tuft ? k_fused_tuft_tma<true> : k_fused_tuft_tma<false>;
        launch_pdl(kern, FT.grid, kThreads, FT.smem, s, A);
    } else {
        uint64_t want = (A.n_units + kWarps - 1) / kWarps;
        uint64_t cap = (uint64_t)F.sms * 8;
        unsigned grid = (unsigned)std::max<uint64_t>(1, std::min(want, cap));
        if (tuft)
            launch_pdl(k_fused_tuft<true>, grid, kWarps * 32, 0, s, A);
        else
            launch_pdl(k_fused_tuft<false>, grid, kWarps * 32, 0, s, A);
    }
}

// ---------------------------------------------------------- batched form --
int prepare_fused_batch(FusedBatch& B, const std::vector<FusedJob>& jobs, const BatchShape& shape) {
    free_fused_batch(B);
    B = FusedBatch{};
    if (jobs.empty()) return BM_OK;
    const bool tuft = jobs[0].L->kind == BM_LYR_PYRAMIDAL;
    uint32_t sms = 148;
    for (const FusedJob& J : jobs) {
        const FusedTuft& FT = J.F->t[J.layer][J.t];
        if (!FT.ok || !FT.tiled || !FT.gidx || (J.L->kind == BM_LYR_PYRAMIDAL) != tuft) return BM_OK;
        sms = (uint32_t)J.F->sms;
    }
    auto kern = tuft ? k_fused_tuft_batch<true> : k_fused_tuft_batch<false>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem);
    // Jobs of one stage geometry share launches (a launch's ring is uniform,
    // and jobs with smaller stages then keep three CTAs per SM).
    std::vector<uint32_t> strides;
    for (const FusedJob& J : jobs) {
        const uint32_t st = J.F->t[J.layer][J.t].stage_stride;
        if (std::find(strides.begin(), strides.end(), st) == strides.end()) strides.push_back(st);
    }
    std::sort(strides.begin(), strides.end());
    for (uint32_t stride : strides) {
        std::vector<const FusedJob*> cls;
        uint32_t halo = 0;
        for (const FusedJob& J : jobs) {
            const FusedTuft& FT = J.F->t[J.layer][J.t];
            if (FT.stage_stride != stride) continue;
            cls.push_back(&J);
            halo = std::max(halo, ((FT.nrec * FT.fsz + 127) / 128) * 128);
        }
        uint32_t nst = ring_stages(stride, halo, shape.max_stages ? std::max<uint32_t>(2, std::min<uint32_t>(4, shape.max_stages)) : 4);
        while (nst > 2 && 128 + (uint64_t)nst * stride + halo > kMaxSmem) nst--;
        const uint64_t ring_off = halo;
        const uint64_t smem = std::max<uint64_t>(32768, ring_off + 128 + (uint64_t)nst * stride);
        if (smem > kMaxSmem) {
            free_fused_batch(B);
            return BM_OK;
        }
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, (size_t)smem) != cudaSuccess)
            per_sm = 1;
        cudaGetLastError();
        if (shape.ctas_per_sm && (int)shape.ctas_per_sm < per_sm) per_sm = (int)shape.ctas_per_sm;
        for (size_t j0 = 0; j0 < cls.size(); j0 += kMaxBatchJobs) {
            auto* P = new (std::nothrow) BatchParams;
            if (!P) {
                free_fused_batch(B);
                return set_err(BM_ERR_OOM, "host allocation failed");
            }
            std::memset(P, 0, sizeof *P);
            const size_t n = std::min<size_t>(kMaxBatchJobs, cls.size() - j0);
            uint32_t total = 0;
            for (size_t j = 0; j < n; j++) {
                const FusedJob& J = *cls[j0 + j];
                make_args(P->jobs[j], *J.F, J.axns, J.slices, *J.L, J.layer, J.t, J.ctl, J.ssc_soma);
                P->jobs[j].nst = nst;
                P->jobs[j].stage_stride = stride;
                P->jobs[j].ring_off = (uint32_t)ring_off;
                P->tile0[j] = total;
                total += P->jobs[j].n_tiles;
            }
            P->tile0[n] = total;
            P->n_jobs = (uint32_t)n;
            P->nst = nst;
            P->ring_off = (uint32_t)ring_off;
            B.params.push_back(P);
            B.grids.push_back((uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(total, (uint64_t)sms * std::max(per_sm, 1))));
            B.smems.push_back((uint32_t)smem);
            B.n_tiles += total;
        }
    }
    B.ok = true;
    B.tuft = tuft;
    B.n_jobs = (uint32_t)jobs.size();
    return BM_OK;
}

uint32_t fused_batch_stages(const void* params) { return ((const BatchParams*)params)->nst; }

void launch_fused_batch(const FusedBatch& B, cudaStream_t s) {
    if (!B.ok || !B.n_tiles) return;
    auto kern = B.tuft ? k_fused_tuft_batch<true> : k_fused_tuft_batch<false>;
    for (size_t k = 0; k < B.params.size(); k++)
        launch_pdl(kern, B.grids[k], kThreads, B.smems[k], s, *(const BatchParams*)B.params[k]);
}

void free_fused_batch(FusedBatch& B) {
    for (void* p : B.params) delete (BatchParams*)p;
    B.params.clear();
    B.grids.clear();
    B.smems.clear();
    B.ok = false;
}

}  // namespace bm
