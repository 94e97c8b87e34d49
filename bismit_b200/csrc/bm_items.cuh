// bm_items.cuh -- the per-item bodies of the per-stage kernels: one synapse,
// dendrite, cell or column each. The one-area kernels (bm_plain.cu) and the
// batched kernels (bm_batch.cu) both call these, so a batched stage computes
// exactly the bytes of the one-area stage.
#pragma once
#include "bm_dev.cuh"

namespace bm {

// layer_cycle_syns_wow[_vec4], cl/syns.cl:179-388; synapse i of tuft t.
__device__ __forceinline__ void syn_cycle_item(const uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices,
                                               const DevLayer& L, uint32_t t, uint64_t i) {
    const DevTuft& T = L.tft[t];
    uint32_t cell = (uint32_t)(i / T.spt);
    uint32_t cols = L.v_size * L.u_size;
    uint32_t rem = cell % cols;
    uint32_t v = rem / L.u_size, u = rem % L.u_size;
    uint64_t si = T.syn_idz + i;
    uint8_t slc = L.buf[BM_BUF_SYN_SRC_SLC_IDS][si];
    int vo = (int8_t)L.buf[BM_BUF_SYN_SRC_COL_V_OFFS][si];
    int uo = (int8_t)L.buf[BM_BUF_SYN_SRC_COL_U_OFFS][si];
    SliceRec s = slices[slc];
    bool safe;
    uint32_t ai = axn_idx(s, v, vo, u, uo, (T.spt & 3) == 0, safe);
    uint8_t a = safe ? axns[ai] : (uint8_t)0;
    L.buf[BM_BUF_SYN_STATES][si] = syn_fire(a);
}

// den_cycle_tft, cl/bismit.cl:695-747; dendrite d of tuft t.
__device__ __forceinline__ void den_cycle_item(const DevLayer& L, uint32_t t, int32_t rnd, uint64_t d) {
    const DevTuft& T = L.tft[t];
    const uint8_t* st = L.buf[BM_BUF_SYN_STATES];
    const int8_t* str = (const int8_t*)L.buf[BM_BUF_SYN_STRENGTHS];
    uint64_t s0 = d * T.spd + T.syn_idz;
    int32_t sum = 0, raw = 0;
    for (uint32_t k = 0; k < T.spd; k++) {
        int32_t a = st[s0 + k];
        sum += (str[s0 + k] >= 0) ? a : 0;
        raw += a;
    }
    int active = (uint32_t)sum > T.thresh;
    sum = active ? sum : 0;
    uint64_t di = d + T.den_idz;
    uint32_t seed = ((uint32_t)raw + T.thresh) | (uint32_t)di;
    L.buf[BM_BUF_DEN_ACTIVITIES][di] =
        update_activity(L.buf[BM_BUF_DEN_ACTIVITIES][di], active, rnd, (int32_t)seed, kDendriteActivityDecay);
    L.buf[BM_BUF_DEN_STATES_RAW][di] = (uint8_t)min(raw >> 4, 255);
    L.buf[BM_BUF_DEN_STATES][di] = (uint8_t)min(sum >> 4, 255);
}

// tft_cycle, cl/bismit.cl:755-842; cell c of tuft t.
__device__ __forceinline__ void tft_cycle_item(const DevLayer& L, uint32_t t, uint32_t c) {
    const DevTuft& T = L.tft[t];
    const uint8_t* sraw = L.buf[BM_BUF_DEN_STATES_RAW];
    const uint8_t* sden = L.buf[BM_BUF_DEN_STATES];
    uint64_t d0 = T.den_idz + (uint64_t)c * T.dpt;
    uint32_t best_id = 0, best_raw = 0, best_st = 0, sum = 0;
    for (uint32_t d = 0; d < T.dpt; d++) {
        uint32_t r = sraw[d0 + d], s = sden[d0 + d];
        if (r > best_raw) { best_id = d; best_raw = r; }
        best_st = max(best_st, s);
        sum += s;
    }
    bool is_max = sum >= (1u << (T.mad_l2 + 8));
    uint8_t state = is_max ? (uint8_t)255 : (uint8_t)(sum >> T.mad_l2);
    uint64_t ci = T.cel_idz + c;
    L.buf[BM_BUF_TFT_PREV_BEST_DEN_IDS][ci] = L.buf[BM_BUF_TFT_BEST_DEN_IDS][ci];
    L.buf[BM_BUF_TFT_PREV_BEST_DEN_STATES_RAW][ci] = L.buf[BM_BUF_TFT_BEST_DEN_STATES_RAW][ci];
    L.buf[BM_BUF_TFT_PREV_BEST_DEN_STATES][ci] = L.buf[BM_BUF_TFT_BEST_DEN_STATES][ci];
    L.buf[BM_BUF_TFT_PREV_STATES][ci] = L.buf[BM_BUF_TFT_STATES][ci];
    L.buf[BM_BUF_TFT_BEST_DEN_IDS][ci] = (uint8_t)best_id;
    L.buf[BM_BUF_TFT_BEST_DEN_STATES_RAW][ci] = (uint8_t)best_raw;
    L.buf[BM_BUF_TFT_BEST_DEN_STATES][ci] = (uint8_t)best_st;
    L.buf[BM_BUF_TFT_STATES][ci] = state;
}

// ssc_cycle, cl/bismit.cl:849-884 (soma = the dendrite state buffer).
__device__ __forceinline__ void ssc_cycle_item(const DevLayer& L, uint32_t c) {
    uint8_t* en = L.buf[BM_BUF_CEL_ENERGIES];
    uint8_t* cs = L.buf[BM_BUF_DEN_STATES];
    uint32_t energy = en[c], state = cs[c];
    int active = state != 0;
    int restless = (energy > 191) & active;
    int dark = energy == 255;
    en[c] = (uint8_t)((dark | restless) ? energy - 64 : energy);
    cs[c] = (uint8_t)min(state + (uint32_t)restless * 255u + (uint32_t)dark * 255u, 255u);
}

__device__ __forceinline__ uint8_t* soma_of(const DevLayer& L) {
    return L.kind == BM_LYR_SPINY_STELLATE ? L.buf[BM_BUF_DEN_STATES] : L.buf[BM_BUF_CEL_STATES];
}

// inhib_simple, cl/control.cl:28-191; cell c. Returns the axon it wrote.
// R > 0: the radius fixed at compile time (the neighbourhood loop unrolls, its
// 3R(R+1)+1 loads independent of one another); R == 0: `radius` at run time.
template <int R>
__device__ __forceinline__ uint8_t inhib_simple_cell(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices,
                                                     const DevLayer& L, int radius_rt, int32_t rnd, uint32_t c) {
    const int radius = R > 0 ? R : radius_rt;
    const uint8_t* cs = soma_of(L);
    int vsz = (int)L.v_size, usz = (int)L.u_size;
    int s = (int)(c / (uint32_t)(vsz * usz)), rem = (int)(c % (uint32_t)(vsz * usz));
    int v = rem / usz, u = rem % usz;
    bool safe;
    uint32_t axi = axn_idx(slices[s + L.base_slc], (uint32_t)v, 0, (uint32_t)u, 0, false, safe);
    uint8_t cel_state = safe ? cs[c] : (uint8_t)0;
    int uninhibited = 1;
    int horizon = radius + kInhibHorizOffset;
    int infl_max = horizon * horizon;
#pragma unroll
    for (int vo = -radius; vo <= radius; vo++) {
        int uz = max(-radius, -vo - radius), um = min(radius, -vo + radius);
#pragma unroll
        for (int uo = uz; uo <= um; uo++) {
            int vt = v + (int)(int8_t)vo, ut = u + (int)(int8_t)uo;
            bool ns = (vt >= 0) & (vt < vsz) & (ut >= 0) & (ut < usz);
            uint8_t nei = ns ? cs[(uint32_t)s * (uint32_t)(vsz * usz) + (uint32_t)(vt * usz + ut)] : (uint8_t)0;
            int dist = (abs(vo) + abs(uo) + abs(-vo - uo)) >> 1;
            int dd = dist - kInhibCenterOffset;
            uninhibited &= ((int)cel_state * infl_max) >= ((int)nei * (infl_max - dd * dd));
        }
    }
    const uint8_t out = (uint8_t)(uninhibited * cel_state);
    axns[axi] = out;
    int axon_active = uninhibited & (cel_state != 0);
    uint8_t* act = L.buf[BM_BUF_CEL_ACTIVITIES];
    act[c] = update_activity(act[c], axon_active, rnd, (int32_t)((uint32_t)cel_state | c), kCellActivityDecay);
    return out;
}
__device__ __forceinline__ uint8_t inhib_simple_item(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices,
                                                     const DevLayer& L, int radius, int32_t rnd, uint32_t c) {
    // Radius 4 (the configurations' inhibition radius) has its own copy.
    return radius == 4 ? inhib_simple_cell<4>(axns, slices, L, radius, rnd, c)
                       : inhib_simple_cell<0>(axns, slices, L, radius, rnd, c);
}

// inhib_passthrough, cl/control.cl:194-217 (rnd is left at 0 by bismit's host,
// src/cortex/iinn.rs:56-66,110-116).
__device__ __forceinline__ void inhib_passthrough_item(uint8_t* __restrict__ axns,
                                                       const SliceRec* __restrict__ slices, const DevLayer& L,
                                                       uint32_t c) {
    const uint8_t* cs = soma_of(L);
    uint32_t cols = L.v_size * L.u_size;
    uint32_t s = c / cols, rem = c % cols;
    bool safe;
    uint32_t axi = axn_idx(slices[s + L.base_slc], rem / L.u_size, 0, rem % L.u_size, 0, false, safe);
    uint8_t st = cs[c];
    axns[axi] = st;
    uint8_t* act = L.buf[BM_BUF_CEL_ACTIVITIES];
    act[c] = update_activity(act[c], st != 0, 0, (int32_t)((uint32_t)st | c), kCellActivityDecay);
}

// ssc_mtp_simple + prx_syns__active__mtp_ltd, cl/bismit.cl:888-915, :604-639;
// cell c (seed syn_idz + i with i starting at syn_idz).
__device__ __forceinline__ void ssc_mtp_item(const uint8_t* __restrict__ axns, const DevLayer& L, int32_t rnd,
                                             uint32_t c) {
    if (!axns[L.axn_idz + c]) return;
    uint32_t spt = L.tft[0].spt;
    const uint8_t* st = L.buf[BM_BUF_SYN_STATES];
    int8_t* str = (int8_t*)L.buf[BM_BUF_SYN_STRENGTHS];
    uint32_t syn_idz = c * spt;
    for (uint32_t i = syn_idz; i < syn_idz + spt; i++) {
        int8_t s = str[i];
        int32_t seed = (int32_t)(syn_idz + i);
        if (st[i] != 0) s = (int8_t)(s + rnd_inc(rnd, seed, s, 0x7F));
        else s = (int8_t)(s - rnd_dec(rnd, seed, s, 0x1FF));
        str[i] = s;
    }
}

// pyr_cycle, cl/bismit.cl:961-1022, bound as at src/cortex/pyramidals.rs:149-164
// (first parameter = best_den_states_raw; apical term discarded at :1021).
__device__ __forceinline__ void pyr_cycle_item(const DevLayer& L, uint32_t c) {
    const uint8_t* braw = L.buf[BM_BUF_TFT_BEST_DEN_STATES_RAW];
    const uint8_t* tst = L.buf[BM_BUF_TFT_STATES];
    uint8_t prx = (L.enabled_flags & kDenBasalProximalFlag) ? tst[(uint64_t)L.prx_id * L.cells + c] : 0;
    uint8_t dst = (L.enabled_flags & kDenBasalDistalFlag) ? braw[(uint64_t)L.dst_id * L.cells + c] : 0;
    int active = prx != 0;
    int is_min = (prx <= 3) && active;
    uint8_t prx_c = (uint8_t)((prx >> 2) + is_min);
    uint8_t dst_c = (uint8_t)(active ? (dst >> 1) : 0);
    L.buf[BM_BUF_CEL_STATES][c] = (uint8_t)(prx_c + dst_c);
}

// pyr_output, cl/control.cl:298-314; cell c.
__device__ __forceinline__ void pyr_output_item(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices,
                                                const DevLayer& L, uint32_t c) {
    uint32_t cols = L.v_size * L.u_size;
    uint32_t s = c / cols, rem = c % cols;
    bool safe;
    uint32_t axi = axn_idx(slices[s + L.base_slc], rem / L.u_size, 0, rem % L.u_size, 0, false, safe);
    axns[axi] = soma_of(L)[c];
}

// inhib_intra_column, cl/control.cl:319-352; column col.
__device__ __forceinline__ void intra_column_item(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices,
                                                  const DevLayer& L, uint32_t col) {
    uint32_t cols = L.v_size * L.u_size;
    const uint8_t* cs = soma_of(L);
    uint32_t v = col / L.u_size, u = col % L.u_size;
    uint8_t best = 0;
    for (uint32_t s = 0; s < L.depth; s++) {
        uint8_t st = cs[s * cols + col];
        best = (st >= best) ? st : (uint8_t)0;
    }
    for (uint32_t s = 0; s < L.depth; s++) {
        bool safe;
        uint32_t axi = axn_idx(slices[s + L.base_slc], v, 0, u, 0, false, safe);
        uint8_t st = cs[s * cols + col];
        axns[axi] = (st >= best) ? st : (uint8_t)0;
    }
}

// tft_dst_mtp + dst_syns__active__mtpot_mtdep, cl/bismit.cl:1195-1268, :554-600
// (pr_l2i = 0, dr_l2i = 5: src/cortex/tufts.rs:158-159); cell c of tuft t.
__device__ __forceinline__ void tft_dst_mtp_item(const uint8_t* __restrict__ axns, const DevLayer& L, uint32_t t,
                                                 int32_t rnd, uint32_t c) {
    const DevTuft& T = L.tft[t];
    uint32_t tci = c + (uint32_t)T.cel_idz;
    uint8_t* cfl = L.buf[BM_BUF_CEL_FLAG_SETS];
    uint8_t f = cfl[c];
    int active = axns[L.axn_idz + c] != 0;
    int prev_active = (f & kCelPrevActiveFlag) != 0;
    if (!prev_active && active && L.buf[BM_BUF_TFT_PREV_BEST_DEN_STATES_RAW][tci] != 0) {
        const uint8_t* sfl = L.buf[BM_BUF_SYN_FLAG_SETS];
        int8_t* str = (int8_t*)L.buf[BM_BUF_SYN_STRENGTHS];
        uint32_t syn_idz = (uint32_t)L.buf[BM_BUF_TFT_PREV_BEST_DEN_IDS][tci] * T.spd + c * T.spt + (uint32_t)T.syn_idz;
        // A best-dendrite id written by the caller past the tuft can address
        // beyond the layer's synapses; such a range is skipped.
        uint32_t n = ((uint64_t)syn_idz + T.spd <= L.n_syns) ? T.spd : 0;
        for (uint32_t i = syn_idz; i < syn_idz + n; i++) {
            int8_t s = str[i];
            int32_t seed = (int32_t)(syn_idz + i);
            if (sfl[i] & kSynPrevActiveFlag) s = (int8_t)(s + rnd_inc(rnd, seed, s, 0x7F));
            else s = (int8_t)(s - rnd_dec(rnd, seed, s, 0xFFF));
            str[i] = s;
        }
    }
    cfl[c] = (uint8_t)((f & ~kCelPrevActiveFlag) | (active ? kCelPrevActiveFlag : 0));
}

// ---------------------------------------------------- fused cell steps ----
// The per-cell steps below run several of bismit's stages for one cell (or
// column) in one thread where each stage depends only on that cell's own
// earlier results; learning, whose work is a run of synapses per active cell,
// is shared by the warp (lanes over synapses) so its accesses coalesce. Their
// per-synapse arithmetic is the per-item bodies' above, unchanged.

// tft_set_syn_flags + layer_cycle_syns + den_cycle_tft (+ tft_cycle) for cell c
// of a tuft the fused tuft kernel does not take (e.g. one-synapse dendrites).
// Flags of a synapse are set from its state before the synapse cycle rewrites
// it, as the stage order has it.
__device__ __forceinline__ void tuft_cell_item(const uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices,
                                               const DevLayer& L, uint32_t t, int32_t rnd_den, uint32_t c) {
    const DevTuft& T = L.tft[t];
    uint8_t* fl = L.buf[BM_BUF_SYN_FLAG_SETS];
    const uint8_t* st = L.buf[BM_BUF_SYN_STATES];
    for (uint32_t k = 0; k < T.spt; k++) {
        const uint64_t i = (uint64_t)c * T.spt + k;
        const uint64_t si = T.syn_idz + i;
        fl[si] = (uint8_t)((fl[si] & ~kSynPrevActiveFlag) | (st[si] ? kSynPrevActiveFlag : 0));
        syn_cycle_item(axns, slices, L, t, i);
    }
    for (uint32_t d = 0; d < T.dpt; d++) den_cycle_item(L, t, rnd_den, (uint64_t)c * T.dpt + d);
    if (L.kind == BM_LYR_PYRAMIDAL) tft_cycle_item(L, t, c);
}

// The strength updates of learning, for every learning cell of the warp
// (lanes in `mask`, each with its run of synapses [z, z + n)), the warp sharing
// each run; kLearnRuns runs at a time, all of them loaded before any is
// stored, so their latencies overlap (runs of different cells are disjoint). SSC:
// prx_syns__active__mtp_ltd (cl/bismit.cl:604-639: a synapse is active when
// its state is non-zero, depression mask 0x1FF); else
// dst_syns__active__mtpot_mtdep (cl/bismit.cl:554-600: active when
// SYN_PREV_ACTIVE is set, depression mask 0xFFF). Both seed with the run's
// first index plus the synapse index (the doubled index, :589,592,629,630).
// Learning runs a warp keeps in flight at once: 8 for spiny stellate cells;
// 4 in the pyramidal tail, where more leaves arrays in local memory.
template <bool SSC, int kLearnRuns = SSC ? 8 : 4>
__device__ __forceinline__ void learn_runs_warp(const DevLayer& L, int32_t rnd, unsigned mask, uint32_t z,
                                                uint32_t n, int lane) {
    const uint8_t* act = SSC ? L.buf[BM_BUF_SYN_STATES] : L.buf[BM_BUF_SYN_FLAG_SETS];
    int8_t* str = (int8_t*)L.buf[BM_BUF_SYN_STRENGTHS];
    constexpr int32_t kDecMask = SSC ? 0x1FF : 0xFFF;
    while (mask) {
        uint32_t zk[kLearnRuns], nk[kLearnRuns], nmax = 0;
#pragma unroll
        for (int k = 0; k < kLearnRuns; k++) {
            const int b = mask ? __ffs(mask) - 1 : 0;
            const uint32_t zb = __shfl_sync(0xFFFFFFFFu, z, b), nb = __shfl_sync(0xFFFFFFFFu, n, b);
            zk[k] = zb;
            nk[k] = mask ? nb : 0u;
            nmax = max(nmax, nk[k]);
            mask &= mask - 1;
        }
        for (uint32_t o = (uint32_t)lane; o < nmax; o += 32) {
            int8_t sv[kLearnRuns];
            uint8_t av[kLearnRuns];
#pragma unroll
            for (int k = 0; k < kLearnRuns; k++) {
                if (o < nk[k]) {
                    sv[k] = str[zk[k] + o];
                    av[k] = act[zk[k] + o];
                }
            }
#pragma unroll
            for (int k = 0; k < kLearnRuns; k++) {
                if (o < nk[k]) {
                    const uint32_t i = zk[k] + o;
                    const int32_t seed = (int32_t)(zk[k] + i);
                    const bool on = SSC ? av[k] != 0 : (av[k] & kSynPrevActiveFlag) != 0;
                    int8_t s = sv[k];
                    if (on) s = (int8_t)(s + rnd_inc(rnd, seed, s, 0x7F));
                    else s = (int8_t)(s - rnd_dec(rnd, seed, s, kDecMask));
                    str[i] = s;
                }
            }
        }
    }
}

// Position of the r-th (0-based) set bit of mask (r < popc(mask)): the
// largest q with fewer than r + 1 set bits below it.
__device__ __forceinline__ int nth_set_bit(unsigned mask, uint32_t r) {
    int q = 0;
#pragma unroll
    for (int step = 16; step; step >>= 1) {
        const int t = q + step;
        const unsigned below = t >= 32 ? mask : (mask & ((1u << t) - 1u));
        if ((uint32_t)__popc(below) <= r) q = t;
    }
    return q;
}

// The same updates as learn_runs_warp when every run has the same length
// `len` (a multiple of 8) and starts on a multiple of 8: the runs' 8-synapse
// pieces are dealt out over the lanes, so one pass of the warp covers 256
// synapses (eight 32-synapse runs at once) with 8-byte loads and stores, and
// a warp's learning cells usually take one pass instead of one per 4 runs.
template <bool SSC>
__device__ __forceinline__ void learn_runs_vec(const DevLayer& L, int32_t rnd, unsigned mask, uint32_t z,
                                               uint32_t len, int lane) {
    const uint8_t* act = SSC ? L.buf[BM_BUF_SYN_STATES] : L.buf[BM_BUF_SYN_FLAG_SETS];
    int8_t* str = (int8_t*)L.buf[BM_BUF_SYN_STRENGTHS];
    constexpr int32_t kDecMask = SSC ? 0x1FF : 0xFFF;
    const uint32_t P = len >> 3;   // pieces a run
    const uint32_t total = (uint32_t)__popc(mask) * P;
    for (uint32_t base = 0; base < total; base += 32) {
        const uint32_t p = base + (uint32_t)lane;
        const bool on = p < total;
        const uint32_t r = on ? p / P : 0u;
        const int src = on ? nth_set_bit(mask, r) : 0;
        const uint32_t zr = __shfl_sync(0xFFFFFFFFu, z, src);
        if (!on) continue;
        const uint32_t z0 = zr + (p - r * P) * 8u;
        const uint2 s8 = *(const uint2*)(str + z0);
        const uint2 a8 = *(const uint2*)(act + z0);
        const uint32_t sw[2] = {s8.x, s8.y}, aw[2] = {a8.x, a8.y};
        uint32_t ow[2];
#pragma unroll
        for (int w = 0; w < 2; w++) {
            uint32_t o = 0;
#pragma unroll
            for (int b = 0; b < 4; b++) {
                const uint32_t i = z0 + (uint32_t)(4 * w + b);
                const int32_t seed = (int32_t)(zr + i);
                const uint8_t av = (uint8_t)(aw[w] >> (8 * b));
                const bool on_syn = SSC ? av != 0 : (av & kSynPrevActiveFlag) != 0;
                int8_t s = (int8_t)(sw[w] >> (8 * b));
                if (on_syn) s = (int8_t)(s + rnd_inc(rnd, seed, s, 0x7F));
                else s = (int8_t)(s - rnd_dec(rnd, seed, s, kDecMask));
                o |= (uint32_t)(uint8_t)s << (8 * b);
            }
            ow[w] = o;
        }
        *(uint2*)(str + z0) = make_uint2(ow[0], ow[1]);
    }
}

// Learning runs of a warp (lanes in mask, runs [z, z + len) of one length):
// 8 synapses a lane when every run's strengths and activity bytes start on an
// 8-byte boundary, else learn_runs_warp.
template <bool SSC>
__device__ __forceinline__ void learn_runs(const DevLayer& L, int32_t rnd, unsigned mask, uint32_t z, uint32_t len,
                                           int lane) {
    if (!mask) return;
    const uintptr_t a = (uintptr_t)(L.buf[BM_BUF_SYN_STRENGTHS] + z) |
                        (uintptr_t)((SSC ? L.buf[BM_BUF_SYN_STATES] : L.buf[BM_BUF_SYN_FLAG_SETS]) + z);
    const bool aligned = (len & 7u) == 0 && __all_sync(0xFFFFFFFFu, !((mask >> lane) & 1u) || (a & 7u) == 0);
    if (aligned) learn_runs_vec<SSC>(L, rnd, mask, z, len, lane);
    else learn_runs_warp<SSC>(L, rnd, mask, z, ((mask >> lane) & 1u) ? len : 0u, lane);
}

// inhib_simple for cell c, then ssc_mtp_simple for the warp's cells whose axon
// came out non-zero. The layer's slices must be plain (the axon inhib_simple
// writes for cell c is axns[axn_idz + c], the one ssc_mtp_simple reads). Every
// lane of the warp calls this; `valid` false for lanes past the last cell.
__device__ __forceinline__ void inhib_mtp_warp(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices,
                                               const DevLayer& L, int radius, int32_t rnd_inhib, int32_t rnd_mtp,
                                               bool learn, uint32_t c, bool valid) {
    const uint8_t ax = valid ? inhib_simple_item(axns, slices, L, radius, rnd_inhib, c) : (uint8_t)0;
    if (!learn) return;
    const uint32_t spt = L.tft[0].spt;
    learn_runs<true>(L, rnd_mtp, __ballot_sync(0xFFFFFFFFu, ax != 0), c * spt, spt, threadIdx.x & 31);
}

// pyr_cycle for the cells of column col, then its control (1: inhib_intra_column,
// 2: pyr_output, 0: none), then tft_dst_mtp for every distal tuft in tuft order
// (each one's CEL_PREV_ACTIVE update seen by the next), the warp sharing the
// synapse runs of the cells that learn. The layer's slices must be plain (the
// axon written for cell c is axns[axn_idz + c], the one learning reads).
// Every lane of the warp calls this; `valid` false past the last column.
// Columns up to kTailDepth cells deep keep the column in registers: every
// input is loaded before any result is stored, so the loads overlap.
constexpr uint32_t kTailDepth = 8;

// Cell c of distal tuft T learns (tft_dst_mtp's condition): its synapse run
// [z, z + n), n = 0 when it does not.
__device__ __forceinline__ void dst_mtp_range(const DevLayer& L, const DevTuft& T, uint32_t c, uint8_t f, bool active,
                                              bool valid, uint32_t& z, uint32_t& n) {
    z = 0;
    n = 0;
    const uint32_t tci = c + (uint32_t)T.cel_idz;
    if (valid && !(f & kCelPrevActiveFlag) && active && L.buf[BM_BUF_TFT_PREV_BEST_DEN_STATES_RAW][tci] != 0) {
        z = (uint32_t)L.buf[BM_BUF_TFT_PREV_BEST_DEN_IDS][tci] * T.spd + c * T.spt + (uint32_t)T.syn_idz;
        // A best-dendrite id written by the caller past the tuft can address
        // beyond the layer's synapses; such a range is skipped.
        n = ((uint64_t)z + T.spd <= L.n_syns) ? T.spd : 0;
    }
}

// The same decision from the cell's previous best raw state and id, already
// loaded (so their loads can be issued with the cell's other inputs).
__device__ __forceinline__ void dst_mtp_range_of(const DevLayer& L, const DevTuft& T, uint32_t c, uint8_t f,
                                                 bool active, bool valid, uint8_t praw, uint8_t pid, uint32_t& z,
                                                 uint32_t& n) {
    z = 0;
    n = 0;
    if (valid && !(f & kCelPrevActiveFlag) && active && praw != 0) {
        z = (uint32_t)pid * T.spd + c * T.spt + (uint32_t)T.syn_idz;
        n = ((uint64_t)z + T.spd <= L.n_syns) ? T.spd : 0;
    }
}

// Lanes per column of the cell-parallel tail: the column's cells sit in
// adjacent lanes (a power of two >= depth); 0 when the column is too deep and
// one thread takes the whole column.
__device__ __forceinline__ uint32_t tail_group(uint32_t depth) {
    return depth <= 1 ? 1u : depth <= 2 ? 2u : depth <= 4 ? 4u : depth <= kTailDepth ? 8u : 0u;
}
__host__ __device__ __forceinline__ uint64_t tail_items(uint32_t depth, uint32_t cols) {
    const uint32_t g = depth <= 1 ? 1u : depth <= 2 ? 2u : depth <= 4 ? 4u : depth <= kTailDepth ? 8u : 1u;
    return (uint64_t)cols * g;
}

// Item t of the tail: lane d of column t / G, G = tail_group(depth), or the
// whole column t when the column is deeper than kTailDepth.
__device__ __forceinline__ void pyr_tail_warp(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices,
                                              const DevLayer& L, int ctrl, bool learn, const AreaCtl* ctl,
                                              uint32_t item, bool valid_item, uint32_t tufts = 0) {
    const uint32_t cols = L.v_size * L.u_size;
    const int lane = threadIdx.x & 31;
    uint8_t* cfl = L.buf[BM_BUF_CEL_FLAG_SETS];
    const uint32_t G = tail_group(L.depth);
    if (G) {
        const uint32_t col = item / G, d = item & (G - 1);
        const bool valid = valid_item && col < cols && d < L.depth;
        const uint32_t c = d * cols + col;
        // Tufts the fused tuft kernel does not take, folded in: their four
        // stages for this cell, which the soma reads next.
        for (uint32_t t = 0; tufts && t < L.n_tufts; t++)
            if (((tufts >> t) & 1) && valid) tuft_cell_item(axns, slices, L, t, rnd_at(L.tft[t].rnd_key_den, ctl->cycle), c);
        const bool prx_on = (L.enabled_flags & kDenBasalProximalFlag) != 0;
        const bool dst_on = (L.enabled_flags & kDenBasalDistalFlag) != 0;
        uint8_t prx = 0, dst = 0, f = 0, ax = 0;
        uint8_t praw[BM_MAX_TUFTS] = {}, pid[BM_MAX_TUFTS] = {};   // distal tufts' previous best
        if (valid) {
            prx = prx_on ? L.buf[BM_BUF_TFT_STATES][(uint64_t)L.prx_id * L.cells + c] : (uint8_t)0;
            dst = dst_on ? L.buf[BM_BUF_TFT_BEST_DEN_STATES_RAW][(uint64_t)L.dst_id * L.cells + c] : (uint8_t)0;
            if (learn) {
                f = cfl[c];
#pragma unroll
                for (uint32_t t = 0; t < BM_MAX_TUFTS; t++) {
                    if (t < L.n_tufts && L.tft[t].den_kind == BM_DEN_DISTAL) {
                        const uint32_t tci = c + (uint32_t)L.tft[t].cel_idz;
                        praw[t] = L.buf[BM_BUF_TFT_PREV_BEST_DEN_STATES_RAW][tci];
                        pid[t] = L.buf[BM_BUF_TFT_PREV_BEST_DEN_IDS][tci];
                    }
                }
            }
            if (ctrl == 0) ax = axns[L.axn_idz + c];
        }
        // pyr_cycle, cl/bismit.cl:961-1022 (as pyr_cycle_item).
        const int p_active = prx != 0;
        const int is_min = (prx <= 3) && p_active;
        const uint8_t soma = (uint8_t)((uint8_t)((prx >> 2) + is_min) + (uint8_t)(p_active ? (dst >> 1) : 0));
        if (valid) L.buf[BM_BUF_CEL_STATES][c] = soma;
        if (ctrl == 1) {
            // inhib_intra_column, cl/control.cl:319-352: the column's cells in
            // depth order through the group's lanes.
            const int base = lane & ~(int)(G - 1);
            uint8_t best = 0;
            for (uint32_t k = 0; k < G; k++) {
                const uint8_t st = (uint8_t)__shfl_sync(0xFFFFFFFFu, (uint32_t)soma, base + (int)k);
                if (k < L.depth) best = (st >= best) ? st : (uint8_t)0;
            }
            ax = (soma >= best) ? soma : (uint8_t)0;
        } else if (ctrl == 2) {
            ax = soma;   // pyr_output, cl/control.cl:298-314
        }
        if (valid && ctrl != 0) axns[L.axn_idz + c] = ax;
        if (!learn) return;
#pragma unroll
        for (uint32_t t = 0; t < BM_MAX_TUFTS; t++) {
            if (t >= L.n_tufts) break;
            const DevTuft& T = L.tft[t];
            if (T.den_kind != BM_DEN_DISTAL) continue;
            const int32_t rnd = rnd_at(T.rnd_key_mtp, ctl->cycle);
            uint32_t z, n;
            dst_mtp_range_of(L, T, c, f, ax != 0, valid, praw[t], pid[t], z, n);
            learn_runs<false>(L, rnd, __ballot_sync(0xFFFFFFFFu, n != 0), z, T.spd, lane);
            f = (uint8_t)((f & ~kCelPrevActiveFlag) | (ax ? kCelPrevActiveFlag : 0));
        }
        if (valid) cfl[c] = f;
        return;
    }
    const uint32_t col = item;
    const bool valid = valid_item && col < cols;
    // Deeper columns: the same steps one cell at a time.
    if (valid) {
        for (uint32_t t = 0; tufts && t < L.n_tufts; t++)
            if ((tufts >> t) & 1)
                for (uint32_t d = 0; d < L.depth; d++)
                    tuft_cell_item(axns, slices, L, t, rnd_at(L.tft[t].rnd_key_den, ctl->cycle), d * cols + col);
        for (uint32_t d = 0; d < L.depth; d++) pyr_cycle_item(L, d * cols + col);
        if (ctrl == 1) intra_column_item(axns, slices, L, col);
        else if (ctrl == 2)
            for (uint32_t d = 0; d < L.depth; d++) pyr_output_item(axns, slices, L, d * cols + col);
    }
    if (!learn) return;
    for (uint32_t d = 0; d < L.depth; d++) {
        const uint32_t c = d * cols + col;
        uint8_t f = valid ? cfl[c] : (uint8_t)0;
        const bool active = valid && axns[L.axn_idz + c] != 0;
        for (uint32_t t = 0; t < L.n_tufts; t++) {
            const DevTuft& T = L.tft[t];
            if (T.den_kind != BM_DEN_DISTAL) continue;
            const int32_t rnd = rnd_at(T.rnd_key_mtp, ctl->cycle);
            uint32_t z, n;
            dst_mtp_range(L, T, c, f, active, valid, z, n);
            learn_runs<false>(L, rnd, __ballot_sync(0xFFFFFFFFu, n != 0), z, T.spd, lane);
            f = (uint8_t)((f & ~kCelPrevActiveFlag) | (active ? kCelPrevActiveFlag : 0));
        }
        if (valid) cfl[c] = f;
    }
}

}  // namespace bm
