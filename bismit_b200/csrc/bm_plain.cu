// bm_plain.cu -- the plain CUDA form of bismit's cycle: one kernel per
// reference stage, one area per launch, same stage order as the reference host.
// Each kernel restates the bismit OpenCL kernel it names; the fused stage
// kernels (bm_fused.cu) must produce identical bytes.
#include "bm_kernels.h"

namespace bm {

namespace {

__device__ __forceinline__ uint64_t gtid() { return (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; }

// tft_set_syn_flags, cl/syns.cl:23-33, 16 synapses per thread.
__global__ void k_set_syn_flags(const uint8_t* __restrict__ states, uint8_t* __restrict__ flags, uint64_t n) {
    uint64_t i = gtid() * 16;
    if (i + 16 <= n && ((((uintptr_t)states) | ((uintptr_t)flags)) & 15) == 0) {
        uint4 s = *(const uint4*)(states + i);
        uint4 f = *(const uint4*)(flags + i);
        uint32_t* sp = (uint32_t*)&s;
        uint32_t* fp = (uint32_t*)&f;
#pragma unroll
        for (int w = 0; w < 4; w++) {
            uint32_t x = sp[w];
            uint32_t nz = (((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x) & 0x80808080u;  // 0x80 per nonzero byte
            fp[w] = (fp[w] & 0xEFEFEFEFu) | (nz >> 3);
        }
        *(uint4*)(flags + i) = f;
    } else {
        for (uint64_t k = i; k < n && k < i + 16; k++)
            flags[k] = (uint8_t)((flags[k] & ~kSynPrevActiveFlag) | (states[k] ? kSynPrevActiveFlag : 0));
    }
}

// layer_cycle_syns_wow[_vec4], cl/syns.cl:179-388; one thread per synapse.
__global__ void k_syn_cycle(const uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices,
                            DevLayer L, uint32_t t) {
    const DevTuft& T = L.tft[t];
    uint64_t i = gtid();
    uint64_t n = (uint64_t)L.cells * T.spt;
    if (i >= n) return;
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

// den_cycle_tft, cl/bismit.cl:695-747; one thread per dendrite.
__global__ void k_den_cycle(DevLayer L, uint32_t t, const AreaCtl* ctl) {
    const DevTuft& T = L.tft[t];
    uint64_t d = gtid();
    if (d >= (uint64_t)L.cells * T.dpt) return;
    int32_t rnd = rnd_at(T.rnd_key_den, ctl->cycle);
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

// tft_cycle, cl/bismit.cl:755-842; one thread per cell.
__global__ void k_tft_cycle(DevLayer L, uint32_t t) {
    const DevTuft& T = L.tft[t];
    uint32_t c = (uint32_t)gtid();
    if (c >= L.cells) return;
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
__global__ void k_ssc_cycle(DevLayer L) {
    uint32_t c = (uint32_t)gtid();
    if (c >= L.cells) return;
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

// inhib_simple, cl/control.cl:28-191; one thread per cell.
__global__ void k_inhib_simple(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices, DevLayer L,
                               int radius, uint64_t rnd_key, const AreaCtl* ctl) {
    uint32_t c = (uint32_t)gtid();
    if (c >= L.cells) return;
    int32_t rnd = rnd_at(rnd_key, ctl->cycle);
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
    for (int vo = -radius; vo <= radius; vo++) {
        int uz = max(-radius, -vo - radius), um = min(radius, -vo + radius);
        for (int uo = uz; uo <= um; uo++) {
            int vt = v + (int)(int8_t)vo, ut = u + (int)(int8_t)uo;
            bool ns = (vt >= 0) & (vt < vsz) & (ut >= 0) & (ut < usz);
            uint8_t nei = ns ? cs[(uint32_t)s * (uint32_t)(vsz * usz) + (uint32_t)(vt * usz + ut)] : (uint8_t)0;
            int dist = (abs(vo) + abs(uo) + abs(-vo - uo)) >> 1;
            int dd = dist - kInhibCenterOffset;
            uninhibited &= ((int)cel_state * infl_max) >= ((int)nei * (infl_max - dd * dd));
        }
    }
    axns[axi] = (uint8_t)(uninhibited * cel_state);
    int axon_active = uninhibited & (cel_state != 0);
    uint8_t* act = L.buf[BM_BUF_CEL_ACTIVITIES];
    act[c] = update_activity(act[c], axon_active, rnd, (int32_t)((uint32_t)cel_state | c), kCellActivityDecay);
}

// inhib_passthrough, cl/control.cl:194-217 (rnd is left at 0 by bismit's host,
// src/cortex/iinn.rs:56-66,110-116).
__global__ void k_inhib_passthrough(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices, DevLayer L) {
    uint32_t c = (uint32_t)gtid();
    if (c >= L.cells) return;
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
// one thread per cell (seed syn_idz + i with i starting at syn_idz).
__global__ void k_ssc_mtp_simple(const uint8_t* __restrict__ axns, DevLayer L, const AreaCtl* ctl) {
    uint32_t c = (uint32_t)gtid();
    if (c >= L.cells) return;
    if (!axns[L.axn_idz + c]) return;
    int32_t rnd = rnd_at(L.rnd_key_ssc_mtp, ctl->cycle);
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
__global__ void k_pyr_cycle(DevLayer L) {
    uint32_t c = (uint32_t)gtid();
    if (c >= L.cells) return;
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

// pyr_output, cl/control.cl:298-314.
__global__ void k_pyr_output(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices, DevLayer L) {
    uint32_t c = (uint32_t)gtid();
    if (c >= L.cells) return;
    uint32_t cols = L.v_size * L.u_size;
    uint32_t s = c / cols, rem = c % cols;
    bool safe;
    uint32_t axi = axn_idx(slices[s + L.base_slc], rem / L.u_size, 0, rem % L.u_size, 0, false, safe);
    axns[axi] = soma_of(L)[c];
}

// inhib_intra_column, cl/control.cl:319-352; one thread per column.
__global__ void k_inhib_intra_column(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices, DevLayer L) {
    uint32_t col = (uint32_t)gtid();
    uint32_t cols = L.v_size * L.u_size;
    if (col >= cols) return;
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
// (pr_l2i = 0, dr_l2i = 5: src/cortex/tufts.rs:158-159); one thread per cell.
__global__ void k_tft_dst_mtp(const uint8_t* __restrict__ axns, DevLayer L, uint32_t t, const AreaCtl* ctl) {
    const DevTuft& T = L.tft[t];
    uint32_t c = (uint32_t)gtid();
    if (c >= L.cells) return;
    uint32_t tci = c + (uint32_t)T.cel_idz;
    uint8_t* cfl = L.buf[BM_BUF_CEL_FLAG_SETS];
    uint8_t f = cfl[c];
    int active = axns[L.axn_idz + c] != 0;
    int prev_active = (f & kCelPrevActiveFlag) != 0;
    if (!prev_active && active && L.buf[BM_BUF_TFT_PREV_BEST_DEN_STATES_RAW][tci] != 0) {
        int32_t rnd = rnd_at(T.rnd_key_mtp, ctl->cycle);
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

inline unsigned nblk(uint64_t n, unsigned b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

// ------------------------------------------------------------ launchers ---
void launch_set_syn_flags(const DevLayer& L, cudaStream_t s) {
    uint64_t n = L.n_syns;
    if (!n) return;
    k_set_syn_flags<<<nblk((n + 15) / 16, 256), 256, 0, s>>>(L.buf[BM_BUF_SYN_STATES], L.buf[BM_BUF_SYN_FLAG_SETS], n);
}
void launch_set_syn_flags_tuft(const DevLayer& L, uint32_t t, cudaStream_t s) {
    const DevTuft& T = L.tft[t];
    uint64_t n = (uint64_t)L.cells * T.spt;
    if (!n) return;
    k_set_syn_flags<<<nblk((n + 15) / 16, 256), 256, 0, s>>>(L.buf[BM_BUF_SYN_STATES] + T.syn_idz,
                                                              L.buf[BM_BUF_SYN_FLAG_SETS] + T.syn_idz, n);
}
void launch_syn_cycle_plain(const uint8_t* axns, const SliceRec* slices, const DevLayer& L, uint32_t t,
                            cudaStream_t s) {
    uint64_t n = (uint64_t)L.cells * L.tft[t].spt;
    k_syn_cycle<<<nblk(n, 256), 256, 0, s>>>(axns, slices, L, t);
}
void launch_den_cycle_plain(const DevLayer& L, uint32_t t, const AreaCtl* ctl, cudaStream_t s) {
    uint64_t n = (uint64_t)L.cells * L.tft[t].dpt;
    k_den_cycle<<<nblk(n, 256), 256, 0, s>>>(L, t, ctl);
}
void launch_tft_cycle_plain(const DevLayer& L, uint32_t t, cudaStream_t s) {
    k_tft_cycle<<<nblk(L.cells, 256), 256, 0, s>>>(L, t);
}
void launch_ssc_cycle(const DevLayer& L, cudaStream_t s) {
    k_ssc_cycle<<<nblk(L.cells, 256), 256, 0, s>>>(L);
}
void launch_inhib_simple(uint8_t* axns, const SliceRec* slices, const DevLayer& L, int radius, uint64_t key,
                         const AreaCtl* ctl, cudaStream_t s) {
    k_inhib_simple<<<nblk(L.cells, 128), 128, 0, s>>>(axns, slices, L, radius, key, ctl);
}
void launch_inhib_passthrough(uint8_t* axns, const SliceRec* slices, const DevLayer& L, cudaStream_t s) {
    k_inhib_passthrough<<<nblk(L.cells, 256), 256, 0, s>>>(axns, slices, L);
}
void launch_ssc_mtp_plain(const uint8_t* axns, const DevLayer& L, const AreaCtl* ctl, cudaStream_t s) {
    k_ssc_mtp_simple<<<nblk(L.cells, 128), 128, 0, s>>>(axns, L, ctl);
}
void launch_pyr_cycle_plain(const DevLayer& L, cudaStream_t s) {
    k_pyr_cycle<<<nblk(L.cells, 256), 256, 0, s>>>(L);
}
void launch_pyr_output(uint8_t* axns, const SliceRec* slices, const DevLayer& L, cudaStream_t s) {
    k_pyr_output<<<nblk(L.cells, 256), 256, 0, s>>>(axns, slices, L);
}
void launch_inhib_intra_column_plain(uint8_t* axns, const SliceRec* slices, const DevLayer& L, cudaStream_t s) {
    k_inhib_intra_column<<<nblk((uint64_t)L.v_size * L.u_size, 256), 256, 0, s>>>(axns, slices, L);
}
void launch_tft_dst_mtp_plain(const uint8_t* axns, const DevLayer& L, uint32_t t, const AreaCtl* ctl,
                              cudaStream_t s) {
    k_tft_dst_mtp<<<nblk(L.cells, 128), 128, 0, s>>>(axns, L, t, ctl);
}

}  // namespace bm
