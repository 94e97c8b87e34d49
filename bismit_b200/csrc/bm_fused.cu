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
// Work layout: a warp takes one 512-byte chunk of the tuft's synapse range per
// step (32 lanes x 16 bytes). Each SoA array (source slice, v/u offsets,
// strength, state, flags) is read with one coalesced 16-byte load per lane;
// new states and flags are written the same way. A lane's 16 synapses belong
// to one dendrite (syns_per_den is a power of two >= 16), so dendrite sums
// reduce across syns_per_den/16 lanes with shuffles, and the tuft argmax across
// the cell's lanes (or across chunks when a cell spans several chunks).
//
// The axon gather uses per-lane slice records (scaled cell coordinates and the
// row-major base index) precomputed once per chunk for the tuft's contiguous
// source slices; any other slice id (e.g. written by the caller) takes the
// general per-synapse path, so every i8 offset and u8 slice id is handled
// exactly as in axn_state_3d_safe (cl/bismit.cl:397-418).
#include "bm_fused.h"

#include <algorithm>
#include <cstring>

namespace bm {

namespace {

constexpr int kWarps = 8;            // warps per CTA
constexpr int kMaxRecs = 8;          // contiguous source slices served from records

struct FusedTuftArgs {
    const uint8_t* axns;
    const SliceRec* slices;
    const AreaCtl* ctl;
    const uint8_t* slc;     // tuft-relative synapse arrays
    const int8_t* vofs;
    const int8_t* uofs;
    const int8_t* str;
    uint8_t* st;
    uint8_t* fl;
    uint8_t* den_act;       // tuft-relative dendrite arrays
    uint8_t* den_raw;
    uint8_t* den_st;
    uint8_t* t_pid;         // tuft-relative cell-tuft arrays (pyramidal)
    uint8_t* t_praw;
    uint8_t* t_pst;
    uint8_t* t_ptft;
    uint8_t* t_bid;
    uint8_t* t_braw;
    uint8_t* t_bst;
    uint8_t* t_st;
    uint64_t n_syn;         // synapses in the tuft
    uint64_t n_units;       // chunks (S <= 512) or cells (S > 512)
    uint32_t den_idz;       // first dendrite (layer index) for the activity seed
    uint32_t thresh;
    uint32_t cols, u_size;
    uint32_t S_l2, spd_l2, lpd_l2, lpc_l2;   // log2 of syns/cell-tuft, syns/den, lanes/den, lanes/cell (<= 5)
    uint32_t chunks_per_unit;
    uint32_t mad_l2;
    uint32_t slc0, nrec;    // records cover slice ids slc0 .. slc0 + nrec - 1
    uint32_t vec4;          // bismit's vec4 synapse kernel semantics (spt % 4 == 0)
    uint64_t rnd_key;
};

struct Rec {
    int32_t base;     // idz + vsc * u_size + usc (row-major index of the cell's scaled position)
    int32_t vsc, usc; // scaled position plus mid
    uint32_t dims;    // v_size | u_size << 16
};

__device__ __forceinline__ uint32_t nz_bits(uint32_t x) {
    // 0x80 in every byte of x that is non-zero.
    return (((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x) & 0x80808080u;
}

__device__ __forceinline__ uint8_t gather_general(const FusedTuftArgs& A, uint8_t slc, uint32_t v, uint32_t u,
                                                  int vo, int uo) {
    bool safe;
    uint32_t ai = axn_idx(A.slices[slc], v, vo, u, uo, A.vec4 != 0, safe);
    return safe ? __ldg(A.axns + ai) : (uint8_t)0;
}

template <bool TUFT>
__global__ void __launch_bounds__(kWarps * 32) k_fused_tuft(FusedTuftArgs A) {
    __shared__ Rec recs[kWarps][kMaxRecs][32];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const uint64_t gwarp = (uint64_t)blockIdx.x * kWarps + wib;
    const uint64_t nwarps = (uint64_t)gridDim.x * kWarps;
    const int32_t rnd = rnd_at(A.rnd_key, A.ctl->cycle);
    const uint32_t lpd = 1u << A.lpd_l2;
    const uint32_t lpc = 1u << A.lpc_l2;

    for (uint64_t unit = gwarp; unit < A.n_units; unit += nwarps) {
        // Tuft accumulators across the chunks of one cell (S > 512).
        uint32_t t_key = 0, t_best = 0, t_sum = 0;
        for (uint32_t ch = 0; ch < A.chunks_per_unit; ch++) {
            const uint64_t chunk = unit * A.chunks_per_unit + ch;
            const uint64_t off = chunk * 512 + (uint64_t)lane * 16;
            const bool on = off < A.n_syn;
            const uint32_t cell = (uint32_t)(off >> A.S_l2);
            const uint32_t rem = cell % A.cols;
            const uint32_t v = rem / A.u_size, u = rem % A.u_size;

            // Per-lane slice records for this cell.
            for (uint32_t k = 0; k < A.nrec; k++) {
                SliceRec s = A.slices[A.slc0 + k];
                Rec r;
                r.vsc = (int32_t)((v * (s.z & 0xFF)) >> kSlcSclCoeffL2);
                r.usc = (int32_t)((u * ((s.z >> 8) & 0xFF)) >> kSlcSclCoeffL2);
                r.dims = s.y;
                r.base = (int32_t)s.x + r.vsc * (int32_t)(s.y >> 16) + r.usc;
                recs[wib][k][lane] = r;
            }
            __syncwarp();

            uint32_t sum = 0, raw = 0;
            if (on) {
                const uint4 slc4 = __ldg((const uint4*)(A.slc + off));
                const uint4 vo4 = __ldg((const uint4*)(A.vofs + off));
                const uint4 uo4 = __ldg((const uint4*)(A.uofs + off));
                const uint4 str4 = __ldg((const uint4*)(A.str + off));
                const uint4 st4 = *(const uint4*)(A.st + off);
                const uint4 fl4 = *(const uint4*)(A.fl + off);
                const uint32_t* sw = (const uint32_t*)&slc4;
                const uint32_t* vw = (const uint32_t*)&vo4;
                const uint32_t* uw = (const uint32_t*)&uo4;
                const uint32_t* strw = (const uint32_t*)&str4;
                const uint32_t* stw = (const uint32_t*)&st4;
                const uint32_t* flw = (const uint32_t*)&fl4;
                uint4 nst4, nfl4;
                uint32_t* nstw = (uint32_t*)&nst4;
                uint32_t* nflw = (uint32_t*)&nfl4;
#pragma unroll
                for (int w = 0; w < 4; w++) {
                    nflw[w] = (flw[w] & 0xEFEFEFEFu) | (nz_bits(stw[w]) >> 3);
                    uint32_t out = 0;
#pragma unroll
                    for (int b = 0; b < 4; b++) {
                        const uint32_t slc = (sw[w] >> (8 * b)) & 0xFF;
                        const int vo = (int)(int8_t)(vw[w] >> (8 * b));
                        const int uo = (int)(int8_t)(uw[w] >> (8 * b));
                        const uint32_t k = slc - A.slc0;
                        uint8_t a;
                        if (k < A.nrec) {
                            const Rec r = recs[wib][k][lane];
                            const int vt = r.vsc + vo, ut = r.usc + uo;
                            const bool safe = ((uint32_t)vt < (r.dims & 0xFFFF)) & ((uint32_t)ut < (r.dims >> 16));
                            a = safe ? __ldg(A.axns + (uint32_t)(r.base + vo * (int32_t)(r.dims >> 16) + uo)) : (uint8_t)0;
                        } else {
                            a = gather_general(A, (uint8_t)slc, v, u, vo, uo);
                        }
                        out |= (uint32_t)syn_fire(a) << (8 * b);
                    }
                    nstw[w] = out;
                    const uint32_t neg = (strw[w] >> 7) & 0x01010101u;
                    raw = __dp4a(out, 0x01010101u, raw);
                    sum = __dp4a(out & ~(neg * 0xFFu), 0x01010101u, sum);
                }
                *(uint4*)(A.st + off) = nst4;
                *(uint4*)(A.fl + off) = nfl4;
            }
            __syncwarp();

            // Dendrite sums across the dendrite's lanes.
            for (uint32_t m = 1; m < lpd; m <<= 1) {
                sum += __shfl_xor_sync(0xFFFFFFFFu, sum, m);
                raw += __shfl_xor_sync(0xFFFFFFFFu, raw, m);
            }
            uint32_t d_raw = 0, d_st = 0;
            const bool lead = on && (lane & (lpd - 1)) == 0;
            const uint64_t den = off >> A.spd_l2;   // dendrite id within the tuft
            if (lead) {
                const int active = sum > A.thresh;
                const uint32_t s2 = active ? sum : 0u;
                const uint32_t di = (uint32_t)den + A.den_idz;
                const uint32_t seed = (raw + A.thresh) | di;
                A.den_act[den] = update_activity(A.den_act[den], active, rnd, (int32_t)seed, kDendriteActivityDecay);
                d_raw = min(raw >> 4, 255u);
                d_st = min(s2 >> 4, 255u);
                A.den_raw[den] = (uint8_t)d_raw;
                A.den_st[den] = (uint8_t)d_st;
            }
            if (TUFT) {
                // Argmax of the raw state with the first (lowest) dendrite winning
                // ties: maximise (raw << 16 | (0xFFFF - id)).
                const uint32_t den_in_cell = (uint32_t)(den & ((1u << (A.S_l2 - A.spd_l2)) - 1));
                uint32_t key = lead ? ((d_raw << 16) | (0xFFFFu - den_in_cell)) : 0u;
                uint32_t best = d_st, tot = d_st;
                for (uint32_t m = lpd; m < lpc; m <<= 1) {
                    key = max(key, __shfl_xor_sync(0xFFFFFFFFu, key, m));
                    best = max(best, __shfl_xor_sync(0xFFFFFFFFu, best, m));
                    tot += __shfl_xor_sync(0xFFFFFFFFu, tot, m);
                }
                t_key = max(t_key, key);
                t_best = max(t_best, best);
                t_sum += tot;
                if (ch + 1 == A.chunks_per_unit && on && (lane & (lpc - 1)) == 0) {
                    const uint32_t c = cell;
                    const uint32_t best_raw = t_key >> 16;
                    const uint32_t best_id = best_raw ? (0xFFFFu - (t_key & 0xFFFFu)) : 0u;
                    const bool is_max = t_sum >= (1u << (A.mad_l2 + 8));
                    const uint8_t tst = is_max ? (uint8_t)255 : (uint8_t)(t_sum >> A.mad_l2);
                    A.t_pid[c] = A.t_bid[c];
                    A.t_praw[c] = A.t_braw[c];
                    A.t_pst[c] = A.t_bst[c];
                    A.t_ptft[c] = A.t_st[c];
                    A.t_bid[c] = (uint8_t)best_id;
                    A.t_braw[c] = (uint8_t)best_raw;
                    A.t_bst[c] = (uint8_t)t_best;
                    A.t_st[c] = tst;
                }
            }
        }
    }
}

inline int ilog2(uint64_t x) {
    int l = 0;
    while ((1ull << l) < x) l++;
    return l;
}
inline bool pow2(uint64_t x) { return x && !(x & (x - 1)); }

}  // namespace

int prepare_fused(FusedArea& F, const bm_area_plan& P, std::string* err) {
    (void)err;
    int dev = 0;
    cudaGetDevice(&dev);
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
    F.sms = sms;
    for (uint32_t i = 0; i < P.n_layers; i++) {
        const bm_layer_plan& L = P.layers[i];
        bool aligned = true;
        for (int k = 0; k < BM_BUF_COUNT; k++)
            if (L.buf_off[k] != UINT64_MAX && (L.buf_off[k] % 16)) aligned = false;
        for (uint32_t t = 0; t < L.n_tufts; t++) {
            const bm_tuft_plan& T = L.tufts[t];
            uint32_t spd = T.syns_per_den, dpt = T.dens_per_tft;
            F.tuft_ok[i][t] = aligned && pow2(spd) && spd >= 16 && spd <= 512 && pow2(dpt) && (T.syn_idz % 16) == 0;
            // Slice records serve the pool's distinct slices when their ids are
            // contiguous and spatial (mid 0, where bismit's scalar and vec4 index
            // forms agree); anything else takes the general per-synapse path.
            uint32_t lo = 255, hi = 0;
            for (uint32_t k = 0; k < T.n_src_uniq; k++) {
                lo = std::min<uint32_t>(lo, T.src_uniq_slc_ids[k]);
                hi = std::max<uint32_t>(hi, T.src_uniq_slc_ids[k]);
            }
            uint32_t nrec = (T.n_src_uniq && hi - lo + 1 <= (uint32_t)kMaxRecs) ? hi - lo + 1 : 0;
            for (uint32_t k = 0; k < nrec; k++)
                if (P.slc_v_mid[lo + k] || P.slc_u_mid[lo + k]) nrec = 0;
            F.slc0[i][t] = nrec ? lo : 0;
            F.nrec[i][t] = nrec;
        }
    }
    return BM_OK;
}

void free_fused(FusedArea& F) { (void)F; }

void launch_fused_tuft(const FusedArea& F, const uint8_t* axns, const SliceRec* slices, const DevLayer& L,
                       uint32_t layer, uint32_t t, const AreaCtl* ctl, cudaStream_t s) {
    const DevTuft& T = L.tft[t];
    FusedTuftArgs A;
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
    A.den_act = L.buf[BM_BUF_DEN_ACTIVITIES] + T.den_idz;
    A.den_raw = L.buf[BM_BUF_DEN_STATES_RAW] + T.den_idz;
    A.den_st = L.buf[BM_BUF_DEN_STATES] + T.den_idz;
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
    A.S_l2 = ilog2(S);
    A.spd_l2 = ilog2(T.spd);
    A.lpd_l2 = A.spd_l2 - 4;
    A.lpc_l2 = std::min<uint32_t>(A.S_l2 - 4, 5);
    A.chunks_per_unit = S > 512 ? (uint32_t)(S / 512) : 1u;
    const uint64_t n_chunks = (A.n_syn + 511) / 512;
    A.n_units = S > 512 ? (uint64_t)L.cells : n_chunks;
    A.mad_l2 = T.mad_l2;
    A.slc0 = F.slc0[layer][t];
    A.nrec = F.nrec[layer][t];
    A.vec4 = (T.spt & 3) == 0;
    A.rnd_key = T.rnd_key_den;
    uint64_t want = (A.n_units + kWarps - 1) / kWarps;
    uint64_t cap = (uint64_t)F.sms * 8;
    unsigned grid = (unsigned)std::max<uint64_t>(1, std::min(want, cap));
    if (tuft)
        k_fused_tuft<true><<<grid, kWarps * 32, 0, s>>>(A);
    else
        k_fused_tuft<false><<<grid, kWarps * 32, 0, s>>>(A);
}

}  // namespace bm
