/*
 * bm_oracle.c -- CPU oracle for the bismit cortical cycle (TEST INFRASTRUCTURE).
 *
 * Used only as the checker by tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg; nothing in the product library links or calls it.
 *
 * Every function restates one piece of bismit and cites the reference lines it
 * follows (paths relative to the bismit repository). Integer semantics follow
 * OpenCL C on a GPU: 32-bit two's-complement wrap-around, arithmetic right
 * shift of negative ints, plain (non-saturating) narrowing to u8/i8.
 */
#include "bm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Reference constants: cl/bismit.cl:11-22, cl/control.cl:6-13, src/cmn/mod.rs:321-336. */
#define SYNAPSE_AXON_BIAS_LOG2          1
#define DENDRITE_ACTIVITY_DECAY_FACTOR  1536
#define CELL_ACTIVITY_DECAY_FACTOR      768
#define INHIB_INFL_CENTER_OFFSET        1
#define INHIB_INFL_HORIZ_OFFSET         3
#define SLC_SCL_COEFF_L2                4
#define CEL_PREV_ACTIVE_FLAG            0x08
#define SYN_PREV_ACTIVE_FLAG            0x10
#define DEN_BASAL_PROXIMAL_FLAG         0x01
#define DEN_BASAL_DISTAL_FLAG           0x02
#define DEN_APICAL_DISTAL_FLAG          0x04
#define BMO_REGROW_PERIOD               201    /* SYNAPSE_REGROWTH_INTERVAL (200, src/cmn/mod.rs:234) + the resetting cycle */
#define BMO_STRENGTH_FLOOR              (-25)  /* SYNAPSE_STRENGTH_FLOOR, src/cmn/mod.rs:233 */

/* ------------------------------------------------------------ helpers ---- */
static inline int32_t shl32(int32_t x, int n) { return (int32_t)((uint32_t)x << n); }
/* gcc defines >> on negative signed ints as an arithmetic shift. */
static inline int32_t asr32(int32_t x, int n) { return x >> n; }
static inline int iabs(int x) { return x < 0 ? -x : x; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int imin(int a, int b) { return a < b ? a : b; }

static inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

/* The per-launch random value. It replaces bismit's host draws
 * `rng.gen::<i32>()` (src/cortex/dendrites.rs:198, src/cortex/tufts.rs:312,
 * src/cortex/spiny_stellates.rs:259, src/cortex/iinn.rs:113) with a seeded,
 * counter-based stream keyed by (area, layer, role, tuft, cycle). */
int32_t bmo_rnd(uint64_t seed, uint32_t area_id, uint32_t layer_id, uint32_t role,
                uint32_t tft_id, uint64_t cycle) {
    uint64_t key = ((uint64_t)area_id << 40) ^ ((uint64_t)layer_id << 32) ^
                   ((uint64_t)role << 24) ^ ((uint64_t)tft_id << 16);
    uint64_t x = splitmix64(splitmix64(seed) + key);
    x = splitmix64(x + cycle);
    return (int32_t)(uint32_t)(x >> 32);
}

/* rnd_mix, cl/bismit.cl:426-431. */
static inline int32_t rnd_mix(int32_t rnd_a, int32_t seed) {
    seed ^= shl32(seed ^ rnd_a, 13);
    seed ^= asr32(seed, 17);
    seed ^= shl32(seed, 5);
    return seed;
}

/* rnd_inc / rnd_dec, cl/bismit.cl:447-469 (abs of a char is its magnitude). */
static inline int rnd_inc(int32_t rnd_a, int32_t seed, int8_t val, int32_t lr_mask) {
    return (rnd_mix(rnd_a, seed) & lr_mask) > (iabs(val) + (lr_mask - 0x7f));
}
static inline int rnd_dec(int32_t rnd_a, int32_t seed, int8_t val, int32_t lr_mask) {
    int val_is_max = val == 127;
    return (rnd_mix(rnd_a, seed) & lr_mask) > ((iabs(val) - val_is_max) + (lr_mask - 0x7f));
}

/* lshft_mask, cl/bismit.cl:473-475: (0x7F << l2i) with the low l2i bits set. */
static inline int32_t lr_mask_of(int l2i) {
    int32_t m = 0x7F << l2i;
    for (int i = 0; i < l2i; i++) m |= (1 << i);
    return m;
}

/* rnd_inc_u, cl/bismit.cl:482-484; rnd_0xFFFF :525-527. */
static inline int rnd_inc_u(int32_t rnd_a, int32_t seed, uint8_t val) {
    return (rnd_mix(rnd_a, seed) & 0xFF) > val;
}
static inline int rnd_0xFFFF(int32_t rnd, int32_t seed, uint16_t cutoff) {
    return (rnd_mix(rnd, seed) & 0xFFFF) < cutoff;
}

/* update_activity_rating, cl/bismit.cl:531-540. */
static inline uint8_t update_activity_rating(uint8_t act, int is_active, int32_t rnd,
                                             int32_t seed, uint16_t decay) {
    act = (uint8_t)(act + (rnd_inc_u(rnd, seed, act) & is_active));
    act = (uint8_t)(act - (rnd_0xFFFF(rnd, shl32(seed, 1), decay) & (act > 0)));
    return act;
}

/* syn_fire, cl/syns.cl:2-4. */
static inline uint8_t syn_fire(uint8_t a) {
    return (uint8_t)(((a != 0) << 7) + (a >> SYNAPSE_AXON_BIAS_LOG2));
}

/* Axon index and bounds of axn_idx_3d_unsafe (cl/bismit.cl:323-363). The
 * scalar form adds the slice mid to the i8 offset in an i8 (wrapping); the
 * vec4 form (:366-391) adds it in int. bismit launches the vec4 synapse kernel
 * when syns_per_tft % 4 == 0 (src/cortex/synapses.rs:261-286). */
static inline uint32_t axn_idx(const bm_area_plan* P, uint8_t slc, uint32_t v_id,
                               int8_t v_ofs_c, uint32_t u_id, int8_t u_ofs_c, int vec4,
                               int* safe) {
    int v_size = (int)P->slc_v_size[slc], u_size = (int)P->slc_u_size[slc];
    int v_ofs, u_ofs;
    if (vec4) {
        v_ofs = (int)v_ofs_c + (int)P->slc_v_mid[slc];
        u_ofs = (int)u_ofs_c + (int)P->slc_u_mid[slc];
    } else {
        v_ofs = (int8_t)(uint8_t)((int)v_ofs_c + (int)P->slc_v_mid[slc]);
        u_ofs = (int8_t)(uint8_t)((int)u_ofs_c + (int)P->slc_u_mid[slc]);
    }
    int v_sc = (int)((v_id * P->slc_v_scale[slc]) >> SLC_SCL_COEFF_L2);
    int u_sc = (int)((u_id * P->slc_u_scale[slc]) >> SLC_SCL_COEFF_L2);
    int vt = v_sc + v_ofs, ut = u_sc + u_ofs;
    *safe = (vt >= 0) & (vt < v_size) & (ut >= 0) & (ut < u_size);
    return P->slc_axn_idz[slc] + (uint32_t)(vt * u_size + ut);
}

/* axn_state_3d_safe[_vec4], cl/bismit.cl:397-418. */
static inline uint8_t axn_state_safe(const bm_area_plan* P, const uint8_t* axns, uint8_t slc,
                                     uint32_t v, int8_t vo, uint32_t u, int8_t uo, int vec4) {
    int safe;
    uint32_t idx = axn_idx(P, slc, v, vo, u, uo, vec4, &safe);
    return safe ? axns[idx] : 0;
}

uint32_t bmo_axn_idx_scl(const bm_area_plan* P, uint8_t slc, uint32_t v, int8_t v_ofs,
                         uint32_t u, int8_t u_ofs, int* safe) {
    return axn_idx(P, slc, v, v_ofs, u, u_ofs, 0, safe);
}
uint32_t bmo_axn_idx_vec4(const bm_area_plan* P, uint8_t slc, int32_t v, int8_t v_ofs,
                          int32_t u, int8_t u_ofs, int* safe) {
    return axn_idx(P, slc, (uint32_t)v, v_ofs, (uint32_t)u, u_ofs, 1, safe);
}

/* ----------------------------------------------------------- layer view -- */
typedef struct {
    const bm_layer_plan* L;
    uint8_t* b[BM_BUF_COUNT];
} lview;

static void view(const bm_layer_plan* L, uint8_t* slab, lview* v) {
    v->L = L;
    for (int k = 0; k < BM_BUF_COUNT; k++)
        v->b[k] = (L->buf_off[k] == UINT64_MAX) ? NULL : slab + L->buf_off[k];
}

/* ------------------------------------------------------------- kernels --- */

/* tft_set_syn_flags, cl/syns.cl:23-33, over every synapse of the layer. */
static void k_set_syn_flags(lview* V) {
    uint8_t* st = V->b[BM_BUF_SYN_STATES];
    uint8_t* fl = V->b[BM_BUF_SYN_FLAG_SETS];
    int64_t n = (int64_t)V->L->n_syns;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        uint8_t f = (uint8_t)(fl[i] & ~SYN_PREV_ACTIVE_FLAG);
        fl[i] = (uint8_t)(f | ((st[i] != 0) ? SYN_PREV_ACTIVE_FLAG : 0));
    }
}

/* layer_cycle_syns_wow[_vec4], cl/syns.cl:179-388: every synapse of one tuft,
 * syn_idx = cel_idx * syns_per_tft + tft_syn_idz + k. */
static void k_syn_cycle(const bm_area_plan* P, const uint8_t* axns, lview* V, const bm_tuft_plan* T) {
    const bm_layer_plan* L = V->L;
    const uint8_t* slc = V->b[BM_BUF_SYN_SRC_SLC_IDS];
    const int8_t* vo = (const int8_t*)V->b[BM_BUF_SYN_SRC_COL_V_OFFS];
    const int8_t* uo = (const int8_t*)V->b[BM_BUF_SYN_SRC_COL_U_OFFS];
    uint8_t* st = V->b[BM_BUF_SYN_STATES];
    uint32_t spt = T->syns_per_tft;
    int vec4 = (spt % 4) == 0;
    int64_t cells = (int64_t)L->cells;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < cells; c++) {
        uint32_t cols = L->v_size * L->u_size;
        uint32_t rem = (uint32_t)(c % cols);
        uint32_t v = rem / L->u_size, u = rem % L->u_size;
        uint64_t base = (uint64_t)c * spt + T->syn_idz;
        for (uint32_t k = 0; k < spt; k++) {
            uint64_t i = base + k;
            st[i] = syn_fire(axn_state_safe(P, axns, slc[i], v, vo[i], u, uo[i], vec4));
        }
    }
}

/* den_cycle_tft, cl/bismit.cl:695-747. */
static void k_den_cycle(lview* V, const bm_tuft_plan* T, int32_t rnd) {
    const uint8_t* st = V->b[BM_BUF_SYN_STATES];
    const int8_t* str = (const int8_t*)V->b[BM_BUF_SYN_STRENGTHS];
    uint8_t* act = V->b[BM_BUF_DEN_ACTIVITIES];
    uint8_t* sraw = V->b[BM_BUF_DEN_STATES_RAW];
    uint8_t* sden = V->b[BM_BUF_DEN_STATES];
    uint32_t spd = T->syns_per_den, thr = T->den_threshold;
    int64_t n_dens = (int64_t)V->L->cells * T->dens_per_tft;
#pragma omp parallel for schedule(static)
    for (int64_t d = 0; d < n_dens; d++) {
        uint64_t s0 = (uint64_t)d * spd + T->syn_idz;
        int32_t sum = 0, raw = 0;
        for (uint32_t k = 0; k < spd; k++) {
            int8_t s = str[s0 + k];
            uint8_t a = st[s0 + k];
            sum += (s >= 0) * (int32_t)a;
            raw += a;
        }
        int active = (uint32_t)sum > thr;
        sum = active * sum;
        uint64_t di = (uint64_t)d + T->den_idz;
        uint32_t seed = ((uint32_t)raw + thr) | (uint32_t)di;
        act[di] = update_activity_rating(act[di], active, rnd, (int32_t)seed,
                                         DENDRITE_ACTIVITY_DECAY_FACTOR);
        int r4 = raw >> 4, s4 = sum >> 4;
        sraw[di] = (uint8_t)(r4 > 255 ? 255 : r4);
        sden[di] = (uint8_t)(s4 > 255 ? 255 : s4);
    }
}

/* tft_cycle, cl/bismit.cl:755-842 (launched per tuft over all cells of the
 * layer, src/cortex/tufts.rs:107-127). */
static void k_tft_cycle(lview* V, const bm_tuft_plan* T) {
    const uint8_t* sraw = V->b[BM_BUF_DEN_STATES_RAW];
    const uint8_t* sden = V->b[BM_BUF_DEN_STATES];
    uint8_t* pid = V->b[BM_BUF_TFT_PREV_BEST_DEN_IDS];
    uint8_t* praw = V->b[BM_BUF_TFT_PREV_BEST_DEN_STATES_RAW];
    uint8_t* pst = V->b[BM_BUF_TFT_PREV_BEST_DEN_STATES];
    uint8_t* ptft = V->b[BM_BUF_TFT_PREV_STATES];
    uint8_t* bid = V->b[BM_BUF_TFT_BEST_DEN_IDS];
    uint8_t* braw = V->b[BM_BUF_TFT_BEST_DEN_STATES_RAW];
    uint8_t* bst = V->b[BM_BUF_TFT_BEST_DEN_STATES];
    uint8_t* tst = V->b[BM_BUF_TFT_STATES];
    uint32_t dpt = T->dens_per_tft, mad = T->max_active_dens_l2;
    int64_t cells = (int64_t)V->L->cells;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < cells; c++) {
        uint64_t d0 = T->den_idz + (uint64_t)c * dpt;
        uint32_t best_id = 0, best_raw = 0, best_st = 0, sum = 0;
        for (uint32_t d = 0; d < dpt; d++) {
            uint32_t r = sraw[d0 + d], s = sden[d0 + d];
            if (r > best_raw) { best_id = d; best_raw = r; }
            if (s > best_st) best_st = s;
            sum += s;
        }
        int is_max = sum >= (1u << (mad + 8));
        uint8_t state = (uint8_t)((uint8_t)(is_max * 255u) + (uint8_t)(!is_max * (sum >> mad)));
        uint64_t ci = T->cel_idz + (uint64_t)c;
        pid[ci] = bid[ci]; praw[ci] = braw[ci]; pst[ci] = bst[ci]; ptft[ci] = tst[ci];
        bid[ci] = (uint8_t)best_id; braw[ci] = (uint8_t)best_raw; bst[ci] = (uint8_t)best_st;
        tst[ci] = state;
    }
}

/* ssc_cycle, cl/bismit.cl:849-884; cel_states is the dendrite state buffer
 * (SpinyStellateLayer::soma, src/cortex/spiny_stellates.rs:78-84). */
static void k_ssc_cycle(lview* V) {
    uint8_t* en = V->b[BM_BUF_CEL_ENERGIES];
    uint8_t* cs = V->b[BM_BUF_DEN_STATES];
    int64_t cells = (int64_t)V->L->cells;
    for (int64_t c = 0; c < cells; c++) {
        uint32_t energy = en[c], state = cs[c];
        int active = state != 0;
        int restless = (energy > 191) & active;
        int dark = energy == 255;
        en[c] = (uint8_t)((dark | restless) ? energy - 64 : energy);
        uint32_t s = state + (uint32_t)restless * 255u + (uint32_t)dark * 255u;
        cs[c] = (uint8_t)(s > 255 ? 255 : s);
    }
}

/* Soma buffer and activities of a host layer (DataCellLayer::soma /
 * activities): SSC soma = dendrite states, pyramidal soma = cell states. */
static uint8_t* soma_of(lview* V) {
    return V->L->kind == BM_LYR_SPINY_STELLATE ? V->b[BM_BUF_DEN_STATES] : V->b[BM_BUF_CEL_STATES];
}

/* inhib_simple, cl/control.cl:28-191. */
static void k_inhib_simple(const bm_area_plan* P, uint8_t* axns, lview* V, int radius, int32_t rnd) {
    const bm_layer_plan* L = V->L;
    const uint8_t* cs = soma_of(V);
    uint8_t* act = V->b[BM_BUF_CEL_ACTIVITIES];
    int vsz = (int)L->v_size, usz = (int)L->u_size;
    int64_t cells = (int64_t)L->cells;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < cells; c++) {
        int s = (int)(c / (vsz * usz)), rem = (int)(c % (vsz * usz));
        int v = rem / usz, u = rem % usz;
        int safe;
        uint32_t axi = axn_idx(P, (uint8_t)(s + L->base_axn_slc), (uint32_t)v, 0, (uint32_t)u, 0, 0, &safe);
        uint8_t cel_state = (uint8_t)(safe * cs[c]);
        int uninhibited = 1;
        int horizon = radius + INHIB_INFL_HORIZ_OFFSET;
        int infl_max = horizon * horizon;
        for (int vo = -radius; vo <= radius; vo++) {
            int vneg = -vo;
            int uz = imax(-radius, vneg - radius), um = imin(radius, vneg + radius);
            for (int uo = uz; uo <= um; uo++) {
                /* cel_state_3d_safe, cl/bismit.cl:285-297 (offsets passed as char). */
                int vo8 = (int8_t)vo, uo8 = (int8_t)uo;
                int vt = v + vo8, ut = u + uo8;
                int nsafe = (vt >= 0) & (vt < vsz) & (ut >= 0) & (ut < usz);
                uint8_t nei = nsafe ? cs[(int64_t)s * vsz * usz + (int64_t)vt * usz + ut] : 0;
                int dist = (iabs(vo) + iabs(uo) + iabs(-vo - uo)) >> 1;
                int dd = dist - INHIB_INFL_CENTER_OFFSET;
                int cel_inf = (int)cel_state * infl_max;
                int nei_inf = (int)nei * (infl_max - dd * dd);
                uninhibited &= cel_inf >= nei_inf;
            }
        }
        axns[axi] = (uint8_t)(uninhibited * cel_state);
        int axon_active = uninhibited & (cel_state != 0);
        act[c] = update_activity_rating(act[c], axon_active, rnd, (int32_t)((uint32_t)cel_state | (uint32_t)c),
                                        CELL_ACTIVITY_DECAY_FACTOR);
    }
}

/* inhib_passthrough, cl/control.cl:194-217. */
static void k_inhib_passthrough(const bm_area_plan* P, uint8_t* axns, lview* V, int32_t rnd) {
    const bm_layer_plan* L = V->L;
    const uint8_t* cs = soma_of(V);
    uint8_t* act = V->b[BM_BUF_CEL_ACTIVITIES];
    for (int64_t c = 0; c < (int64_t)L->cells; c++) {
        uint32_t cols = L->v_size * L->u_size;
        int s = (int)(c / cols), rem = (int)(c % cols);
        int v = rem / (int)L->u_size, u = rem % (int)L->u_size;
        int safe;
        uint32_t axi = axn_idx(P, (uint8_t)(s + L->base_axn_slc), (uint32_t)v, 0, (uint32_t)u, 0, 0, &safe);
        uint8_t st = cs[c];
        axns[axi] = st;
        act[c] = update_activity_rating(act[c], st != 0, rnd, (int32_t)((uint32_t)st | (uint32_t)c),
                                        CELL_ACTIVITY_DECAY_FACTOR);
    }
}

/* ssc_mtp_simple + prx_syns__active__mtp_ltd, cl/bismit.cl:888-915, :604-639.
 * The seed is syn_idz + i with i already starting at syn_idz (doubled). */
static void k_ssc_mtp_simple(const bm_area_plan* P, const uint8_t* axns, lview* V, int32_t rnd) {
    const bm_layer_plan* L = V->L;
    const uint8_t* st = V->b[BM_BUF_SYN_STATES];
    int8_t* str = (int8_t*)V->b[BM_BUF_SYN_STRENGTHS];
    uint32_t spt = L->tufts[0].syns_per_tft;
    const int32_t pr_mask = lr_mask_of(0), dr_mask = lr_mask_of(2);
    int64_t cells = (int64_t)L->cells;
    (void)P;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t c = 0; c < cells; c++) {
        if (!axns[L->axn_idz + (uint32_t)c]) continue;
        uint32_t syn_idz = (uint32_t)c * spt;
        for (uint32_t i = syn_idz; i < syn_idz + spt; i++) {
            int8_t s = str[i];
            int32_t seed = (int32_t)(syn_idz + i);
            int inc = rnd_inc(rnd, seed, s, pr_mask);
            int dec = rnd_dec(rnd, seed, s, dr_mask);
            int active = st[i] != 0;
            s = (int8_t)(s + active * inc);
            s = (int8_t)(s - (!active) * dec);
            str[i] = s;
        }
    }
}

/* pyr_cycle, cl/bismit.cl:961-1022, bound as at src/cortex/pyramidals.rs:149-164:
 * the first parameter receives best_den_states_raw, and the apical term is
 * discarded by the comma operator at :1021. */
static void k_pyr_cycle(lview* V) {
    const bm_layer_plan* L = V->L;
    const uint8_t* braw = V->b[BM_BUF_TFT_BEST_DEN_STATES_RAW];
    const uint8_t* tst = V->b[BM_BUF_TFT_STATES];
    uint8_t* ps = V->b[BM_BUF_CEL_STATES];
    uint32_t cells = L->cells, fl = L->enabled_tft_flags;
    for (uint32_t c = 0; c < cells; c++) {
        int prx_en = (fl & DEN_BASAL_PROXIMAL_FLAG) != 0;
        int dst_en = (fl & DEN_BASAL_DISTAL_FLAG) != 0;
        uint8_t prx = (uint8_t)(prx_en * tst[(uint64_t)L->bsl_prx_tft_id * cells + c]);
        uint8_t dst = (uint8_t)(dst_en * braw[(uint64_t)L->bsl_dst_tft_id * cells + c]);
        int active = prx != 0;
        int is_min = (prx <= 3) && active;
        uint8_t prx_c = (uint8_t)((prx >> 2) + is_min);
        uint8_t dst_c = (uint8_t)(active * (dst >> 1));
        ps[c] = (uint8_t)(prx_c + dst_c);
    }
}

/* pyr_output, cl/control.cl:298-314. */
static void k_pyr_output(const bm_area_plan* P, uint8_t* axns, lview* V) {
    const bm_layer_plan* L = V->L;
    const uint8_t* cs = soma_of(V);
    uint32_t cols = L->v_size * L->u_size;
    for (uint32_t c = 0; c < L->cells; c++) {
        uint32_t s = c / cols, rem = c % cols, v = rem / L->u_size, u = rem % L->u_size;
        int safe;
        uint32_t axi = axn_idx(P, (uint8_t)(s + L->base_axn_slc), v, 0, u, 0, 0, &safe);
        axns[axi] = cs[c];
    }
}

/* inhib_intra_column, cl/control.cl:319-352 (best = (state >= best) * state). */
static void k_inhib_intra_column(const bm_area_plan* P, uint8_t* axns, lview* V) {
    const bm_layer_plan* L = V->L;
    const uint8_t* cs = soma_of(V);
    uint32_t cols = L->v_size * L->u_size;
    for (uint32_t col = 0; col < cols; col++) {
        uint32_t v = col / L->u_size, u = col % L->u_size;
        uint8_t best = 0;
        for (uint32_t s = 0; s < L->depth; s++) {
            uint8_t st = cs[s * cols + col];
            best = (uint8_t)((st >= best) * st);
        }
        for (uint32_t s = 0; s < L->depth; s++) {
            int safe;
            uint32_t axi = axn_idx(P, (uint8_t)(s + L->base_axn_slc), v, 0, u, 0, 0, &safe);
            uint8_t st = cs[s * cols + col];
            axns[axi] = (uint8_t)((st >= best) * st);
        }
    }
}

/* tft_dst_mtp + dst_syns__active__mtpot_mtdep, cl/bismit.cl:1195-1268, :554-600,
 * launched per distal tuft with pr_l2i = 0, dr_l2i = 5 (src/cortex/tufts.rs:151-208). */
static void k_tft_dst_mtp(const uint8_t* axns, lview* V, const bm_tuft_plan* T, int32_t rnd) {
    const bm_layer_plan* L = V->L;
    const uint8_t* pid = V->b[BM_BUF_TFT_PREV_BEST_DEN_IDS];
    const uint8_t* praw = V->b[BM_BUF_TFT_PREV_BEST_DEN_STATES_RAW];
    const uint8_t* sfl = V->b[BM_BUF_SYN_FLAG_SETS];
    uint8_t* cfl = V->b[BM_BUF_CEL_FLAG_SETS];
    int8_t* str = (int8_t*)V->b[BM_BUF_SYN_STRENGTHS];
    const int32_t pr_mask = lr_mask_of(0), dr_mask = lr_mask_of(5);
    uint32_t spd = T->syns_per_den, spt = T->syns_per_tft;
    int64_t cells = (int64_t)L->cells;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t ci = 0; ci < cells; ci++) {
        uint32_t c = (uint32_t)ci;
        uint32_t tci = c + (uint32_t)T->cel_idz;
        uint32_t syn_idz_celtft = c * spt + (uint32_t)T->syn_idz;
        uint8_t f = cfl[c];
        int active = axns[L->axn_idz + c] != 0;
        int prev_active = (f & CEL_PREV_ACTIVE_FLAG) == CEL_PREV_ACTIVE_FLAG;
        int newly = (!prev_active) & active;
        int tft_prev_active = praw[tci] != 0;
        if (newly & tft_prev_active) {
            uint32_t syn_idz = (uint32_t)pid[tci] * spd + syn_idz_celtft;
            /* Out-of-layer ranges (only reachable through caller-written ids) are skipped. */
            uint32_t n = ((uint64_t)syn_idz + spd <= L->n_syns) ? spd : 0;
            for (uint32_t i = syn_idz; i < syn_idz + n; i++) {
                int8_t s = str[i];
                int32_t seed = (int32_t)(syn_idz + i);
                if ((sfl[i] & SYN_PREV_ACTIVE_FLAG) == SYN_PREV_ACTIVE_FLAG)
                    s = (int8_t)(s + rnd_inc(rnd, seed, s, pr_mask));
                else
                    s = (int8_t)(s - rnd_dec(rnd, seed, s, dr_mask));
                str[i] = s;
            }
        }
        f = (uint8_t)(f & ~CEL_PREV_ACTIVE_FLAG);
        f = (uint8_t)(f | (active * CEL_PREV_ACTIVE_FLAG));
        cfl[c] = f;
    }
}

/* ActivitySmoother group centers: gen_grp_centers (src/cortex/smoother.rs:
 * 11-33) with HexGroupCenters (src/cmn/mod.rs:809-917). Lattice k is grown
 * from its start by the six moves of add_surrounds, within [-r, dims + r);
 * centers are returned row-major (the reference keeps them in a hash set;
 * the groups of one lattice are disjoint, so their order does not matter).
 * Writes (v, u) pairs into out (capacity 2 * cap) and the lattice ranges
 * into off[7]; returns -1 on overflow. */
static int smoother_centers(int r, int V, int U, int32_t* out, int cap, int off[7]) {
    const int l = r + 1, s = r, ls = l + s;
    const int mv[6][2] = {{-s, ls}, {l, s}, {ls, -l}, {s, -ls}, {-l, -s}, {-ls, l}};
    const int ofs = (r + 1) / 2;
    const int st[6][2] = {{0, ofs}, {-ofs, ofs}, {-ofs, 0}, {0, -ofs}, {ofs, -ofs}, {ofs, 0}};
    const int W = U + 2 * r, H = V + 2 * r;
    uint8_t* seen = (uint8_t*)calloc((size_t)W * H, 1);
    int* stack = (int*)malloc(sizeof(int) * 2 * (size_t)W * H + 16);
    int n = 0;
    for (int k = 0; k < 6; k++) {
        memset(seen, 0, (size_t)W * H);
        off[k] = n;
        int top = 0;
        if (st[k][0] >= -r && st[k][1] >= -r && st[k][0] < V + r && st[k][1] < U + r) {
            seen[(st[k][0] + r) * W + (st[k][1] + r)] = 1;
            stack[top++] = st[k][0];
            stack[top++] = st[k][1];
        }
        while (top) {
            int cu = stack[--top], cv = stack[--top];
            for (int m = 0; m < 6; m++) {
                int v = cv + mv[m][0], u = cu + mv[m][1];
                if (v < -r || u < -r || v >= V + r || u >= U + r) continue;
                if (seen[(v + r) * W + (u + r)]) continue;
                seen[(v + r) * W + (u + r)] = 1;
                stack[top++] = v;
                stack[top++] = u;
            }
        }
        for (int v = -r; v < V + r; v++)
            for (int u = -r; u < U + r; u++)
                if (seen[(v + r) * W + (u + r)]) {
                    if (n >= cap) { free(seen); free(stack); return -1; }
                    out[2 * n] = v;
                    out[2 * n + 1] = u;
                    n++;
                }
    }
    off[6] = n;
    free(seen);
    free(stack);
    return 0;
}

/* smooth_activity (cl/control.cl:227-295), the six lattices in order (the
 * reference launches every center at once and its work-items race on the
 * energies; lattice order is one of the outcomes that race can give). For
 * each center: scan the hexagon of side r over every slice of the host layer
 * (slice, v offset, u offset), keep the least active in-bounds cell (ties:
 * the later) and the most active (ties: the later); then the least active
 * cell's energy += 1 when below 255, the most active's -= 1 when above 0,
 * both only when the two cells differ and (for the raise) the most active
 * activity is below 255, (for the lowering) above 0. ActivitySmoother::cycle
 * (src/cortex/smoother.rs:154-169) runs it every cycle: its counter is never
 * stored, so `cycle_count & 0xFF == 0` always holds. */
static void k_smooth_activity(lview* V, int r) {
    const bm_layer_plan* L = V->L;
    const int Vs = (int)L->v_size, Us = (int)L->u_size;
    const int cap = 6 * (Vs + 2 * r + 2) * (Us + 2 * r + 2);
    int32_t* c = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)cap);
    int off[7];
    if (smoother_centers(r, Vs, Us, c, cap, off)) { free(c); return; }
    const uint8_t* act = V->b[BM_BUF_CEL_ACTIVITIES];
    uint8_t* en = V->b[BM_BUF_CEL_ENERGIES];
    for (int i = 0; i < off[6]; i++) {
        const int cv = c[2 * i], cu = c[2 * i + 1];
        uint32_t li = 0, mi = 0, la = 255, ma = 0;
        for (uint32_t slc = 0; slc < L->depth; slc++)
            for (int vo = -r; vo <= r; vo++) {
                int uz = imax(-r, -vo - r), um = imin(r, -vo + r);
                for (int uo = uz; uo <= um; uo++) {
                    int v = cv + vo, u = cu + uo;
                    if (v < 0 || v >= Vs || u < 0 || u >= Us) continue;
                    uint32_t idx = slc * (uint32_t)(Vs * Us) + (uint32_t)(v * Us + u);
                    uint32_t a = act[idx];
                    if (a <= la) { li = idx; la = a; }
                    if (a >= ma) { mi = idx; ma = a; }
                }
            }
        int differ = li != mi;
        uint32_t le = en[li];
        en[li] = (uint8_t)(le + (uint32_t)((le < 255) & (ma < 255) & differ));
        uint32_t me = en[mi];
        en[mi] = (uint8_t)(me - (uint32_t)((me > 0) & (ma > 0) & differ));
    }
    free(c);
}

/* retina (cl/filters.cl:34-100) over a (depth, vs, us) grid of input bytes:
 * cell i is off-center when bit 0 of i is set and large when bits 1 and 0
 * differ; get_neighbors_avg (:8-31) sums the hexagon of radius 5 (large) or 3
 * (small) in the cell's slice, a cell outside the grid reading as 0
 * (cel_state_3d_safe, cl/bismit.cl:285-297) but counted all the same. The
 * output goes to slice base_slc + slice at that slice's first axon
 * (get_axn_idz, cl/bismit.cl:117-119) plus the cell's place in the slice. */
static void k_retina(const bm_area_plan* P, const uint8_t* in, uint8_t* out, uint32_t base_slc,
                     uint32_t depth, uint32_t vs, uint32_t us) {
    const uint32_t cols = vs * us;
    for (uint32_t i = 0; i < depth * cols; i++) {
        const uint32_t slc = i / cols, col = i % cols;
        const int v = (int)(col / us), u = (int)(col % us);
        const int off_cen = (int)(i & 1), large = (int)((i & 3) >> 1) ^ off_cen;
        const int r = large ? 5 : 3;
        int sum = 0, count = 0;
        for (int vo = -r; vo <= r; vo++) {
            const int uz = imax(-r, -vo - r), um = imin(r, -vo + r);
            for (int uo = uz; uo <= um; uo++) {
                const int vv = v + vo, uu = u + uo;
                if (vv >= 0 && vv < (int)vs && uu >= 0 && uu < (int)us)
                    sum += in[slc * cols + (uint32_t)(vv * (int)us + uu)];
                count++;
            }
        }
        const int avg = sum / count, center = in[i];
        int st = 0;
        if (off_cen) {
            const int cst = center + 48;   /* RETNAL_THRESHOLD, cl/bismit.cl:19 */
            if (avg > cst) st = avg - cst;
        } else {
            const int nat = avg + 48;
            if (center > nat) st = center - nat;
        }
        out[P->slc_axn_idz[(base_slc + slc) & 0xFF] + col] = (uint8_t)st;
    }
}

static int filters_run(const bm_area_plan* P) {
    return P->n_filter_chains && !(P->settings & BM_SET_BYPASS_FILTERS);
}

/* AxonSpace::intake (src/cortex/axon_space.rs:510-525): every filter of each
 * chain in order, filter k from its buffer to the next one's (output slices
 * from slice 0), the last to the target slices (SensoryFilter::new and
 * ::cycle, src/cortex/sensory_filter.rs:25-110,157-168). */
static void run_filters(const bm_area_plan* P, uint8_t* slab) {
    if (!filters_run(P)) return;
    for (uint32_t k = 0; k < P->n_filter_chains; k++) {
        const bm_filter_chain_plan* c = &P->filter_chains[k];
        for (uint32_t f = 0; f < c->n_filters; f++) {
            const int last = f + 1 == c->n_filters;
            k_retina(P, slab + c->buf_off[f], last ? slab + P->axon_off : slab + c->buf_off[f + 1],
                     last ? c->tar_slc : 0, c->depth, c->v_size, c->u_size);
        }
    }
}

/* Bytes [off, off + len) of a frame of input `input`: a source with a running
 * filter chain goes to the chain's first buffer (SensoryFilter::write,
 * sensory_filter.rs:122-155), the rest straight to the input's axons
 * (axon_space.rs:526-560). */
int bmo_intake(const bm_area_plan* P, uint8_t* slab, uint32_t input, uint32_t off, const uint8_t* data,
               uint32_t len) {
    if (input >= P->n_inputs || off > P->inputs[input].len || len > P->inputs[input].len - off) return -1;
    uint8_t* axns = slab + P->axon_off + P->inputs[input].axn_idz;
    for (uint32_t b = off; b < off + len; b++) {
        uint8_t* dst = axns + b;
        for (uint32_t k = 0; filters_run(P) && k < P->n_filter_chains; k++) {
            const bm_filter_chain_plan* c = &P->filter_chains[k];
            const uint32_t c0 = c->frame_off, c1 = c0 + c->depth * c->v_size * c->u_size;
            if (c->input == input && b >= c0 && b < c1) dst = slab + c->buf_off[0] + (b - c0);
        }
        *dst = data[b - off];
    }
    return 0;
}

/* --------------------------------------------------------- layer steps --- */

/* Control layers hosted on V in (host, exe_order) order
 * (src/cortex/control_cell_layer.rs:21, src/cortex/iinn.rs:105-127,
 * src/cortex/intra_column_inhib.rs:80-92, src/cortex/pyr_outputter.rs:70-80,
 * src/cortex/smoother.rs:154-169). */
static void controls_post(const bm_area_plan* P, uint8_t* axns, lview* V, uint64_t cyc) {
    const bm_layer_plan* L = V->L;
    for (uint32_t k = 0; k < L->n_ctrl; k++) {
        const bm_ctrl_plan* C = &L->ctrl[k];
        switch (C->kind) {
        case BM_LYR_CTRL_INHIB_BASKET:
            if (P->settings & BM_SET_BYPASS_INHIB)
                k_inhib_passthrough(P, axns, V, 0);
            else
                k_inhib_simple(P, axns, V, (int)C->field_radius,
                               bmo_rnd(P->rnd_seed, P->area_id, C->layer_id, BM_RND_INHIB, 0, cyc));
            break;
        case BM_LYR_CTRL_PYR_OUTPUT: k_pyr_output(P, axns, V); break;
        case BM_LYR_CTRL_INTRA_COLUMN: k_inhib_intra_column(P, axns, V); break;
        case BM_LYR_CTRL_SMOOTHER: k_smooth_activity(V, (int)C->field_radius); break;
        default: break;
        }
    }
}

/* Dendrites::cycle (src/cortex/dendrites.rs:191-209) with Synapses::cycle
 * (src/cortex/synapses.rs:363-387) in front. */
static void dens_cycle(const bm_area_plan* P, uint8_t* axns, lview* V, uint64_t cyc) {
    const bm_layer_plan* L = V->L;
    k_set_syn_flags(V);
    for (uint32_t t = 0; t < L->n_tufts; t++) k_syn_cycle(P, axns, V, &L->tufts[t]);
    for (uint32_t t = 0; t < L->n_tufts; t++)
        k_den_cycle(V, &L->tufts[t], bmo_rnd(P->rnd_seed, P->area_id, L->layer_id, BM_RND_DEN_CYCLE, t, cyc));
}

/* SpinyStellateLayer::cycle, src/cortex/spiny_stellates.rs:220-252. */
static void ssc_layer_cycle(const bm_area_plan* P, uint8_t* axns, lview* V, uint64_t cyc) {
    dens_cycle(P, axns, V, cyc);
    k_ssc_cycle(V);
    controls_post(P, axns, V, cyc);
}

/* PyramidalLayer::cycle, src/cortex/pyramidals.rs:297-335 (learning included). */
static void pyr_layer_cycle(const bm_area_plan* P, uint8_t* axns, lview* V, uint64_t cyc) {
    const bm_layer_plan* L = V->L;
    dens_cycle(P, axns, V, cyc);
    for (uint32_t t = 0; t < L->n_tufts; t++) k_tft_cycle(V, &L->tufts[t]);
    k_pyr_cycle(V);
    controls_post(P, axns, V, cyc);
    if (!(P->settings & (BM_SET_DISABLE_LEARNING | BM_SET_DISABLE_PYRS))) {
        for (uint32_t t = 0; t < L->n_tufts; t++)
            if (L->tufts[t].den_kind == BM_DEN_DISTAL)
                k_tft_dst_mtp(axns, V, &L->tufts[t],
                              bmo_rnd(P->rnd_seed, P->area_id, L->layer_id, BM_RND_TFT_DST_MTP, t, cyc));
    }
}

static void layer_learn(const bm_area_plan* P, uint8_t* axns, lview* V, uint64_t cyc) {
    const bm_layer_plan* L = V->L;
    if (L->kind == BM_LYR_SPINY_STELLATE) {
        if (!(P->settings & (BM_SET_DISABLE_LEARNING | BM_SET_DISABLE_SSCS)))
            k_ssc_mtp_simple(P, axns, V,
                             bmo_rnd(P->rnd_seed, P->area_id, L->layer_id, BM_RND_SSC_MTP, 0, cyc));
    } else {
        if (!(P->settings & (BM_SET_DISABLE_LEARNING | BM_SET_DISABLE_PYRS))) {
            for (uint32_t t = 0; t < L->n_tufts; t++)
                if (L->tufts[t].den_kind == BM_DEN_DISTAL)
                    k_tft_dst_mtp(axns, V, &L->tufts[t],
                                  bmo_rnd(P->rnd_seed, P->area_id, L->layer_id, BM_RND_TFT_DST_MTP, t, cyc));
        }
    }
}

static void layer_cycle(const bm_area_plan* P, uint8_t* axns, lview* V, uint64_t cyc) {
    if (V->L->kind == BM_LYR_SPINY_STELLATE) ssc_layer_cycle(P, axns, V, cyc);
    else pyr_layer_cycle(P, axns, V, cyc);
}

static void regrow_layer(const bm_area_plan* P, lview* V, uint64_t cyc);

/* CorticalArea::cycle, src/cortex/cortical_area.rs:716-789 (the samplers
 * excluded), regrowth included. */
static void area_cycle(const bm_area_plan* P, uint8_t* slab, uint64_t cyc) {
    uint8_t* axns = slab + P->axon_off;
    lview V[BM_MAX_LAYERS];
    for (uint32_t l = 0; l < P->n_layers; l++) view(&P->layers[l], slab, &V[l]);
    run_filters(P, slab);
    if (!(P->settings & BM_SET_DISABLE_SSCS)) {
        for (uint32_t k = 0; k < P->n_cycle_order; k++) {
            lview* v = &V[P->cycle_order[k]];
            if (v->L->tags & BM_TAG_SPATIAL) layer_cycle(P, axns, v, cyc);
        }
        for (uint32_t k = 0; k < P->n_cycle_order; k++) {
            lview* v = &V[P->cycle_order[k]];
            if (v->L->tags & BM_TAG_SPATIAL) layer_learn(P, axns, v, cyc);
        }
    }
    if (!(P->settings & BM_SET_DISABLE_PYRS)) {
        for (uint32_t k = 0; k < P->n_cycle_order; k++) {
            lview* v = &V[P->cycle_order[k]];
            if (!(v->L->tags & BM_TAG_SPATIAL)) layer_cycle(P, axns, v, cyc);
        }
    }
    /* CorticalArea::regrow (src/cortex/cortical_area.rs:792-806): every data
     * layer in cycle order, on the cycles the regrowth counter fires (it
     * counts up from 0 and fires, resetting, once it has reached 200). */
    if (!(P->settings & BM_SET_DISABLE_REGROWTH) && cyc % BMO_REGROW_PERIOD == BMO_REGROW_PERIOD - 1)
        for (uint32_t k = 0; k < P->n_cycle_order; k++) regrow_layer(P, &V[P->cycle_order[k]], cyc);
}

int bmo_run(const bm_area_plan* P, uint8_t* slab, const uint8_t* frames, uint64_t frame_len,
            uint32_t n_cycles, uint64_t start_cycle, int n_threads) {
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#else
    (void)n_threads;
#endif
    if (frames && P->n_inputs == 0) return -1;
    if (frames && frame_len != P->inputs[0].len) return -2;
    for (uint32_t k = 0; k < n_cycles; k++) {
        if (frames) bmo_intake(P, slab, 0, 0, frames + (uint64_t)k * frame_len, P->inputs[0].len);
        area_cycle(P, slab, start_cycle + k);
    }
    return 0;
}

/* ----------------------------------------------------------- growth ---- */

/* gen_syn_offs, src/map/syn_src.rs:47-149 (scale: src/cmn/slice_dims.rs:192-194). */
int bmo_gen_syn_offs(int radius, uint32_t v_scale, uint32_t u_scale, int8_t* v_out,
                     int8_t* u_out, int cap) {
    if (radius < 0) return -1;
    int v_rad = (radius * (int)v_scale) >> SLC_SCL_COEFF_L2;
    int u_rad = (radius * (int)u_scale) >> SLC_SCL_COEFF_L2;
    int rmax = v_rad > u_rad ? v_rad : u_rad;
    if (rmax > 127) return -1;
    if (v_scale == 0) return -1;
    int n = 0;
    for (int vo = -v_rad; vo <= v_rad; vo++) {
        int vinv = -vo;
        int a = imax(-v_rad, vinv - v_rad), b = imin(v_rad, vinv + v_rad);
        /* scl_inv_scl: (val * (scl << 3)) / (scl_inv << 3), truncating. */
        int uz = (a * ((int)u_scale << 3)) / ((int)v_scale << 3);
        int un = (b * ((int)u_scale << 3)) / ((int)v_scale << 3) + 1;
        for (int uo = uz; uo < un; uo++) {
            if (vo > 127 || vo < -127 || uo > 127 || uo < -127) return -1;
            if (n >= cap) return -1;
            v_out[n] = (int8_t)vo;
            u_out[n] = (int8_t)uo;
            n++;
        }
    }
    return n;
}

/* The per-dendrite growth stream: word k of dendrite d of (layer, tuft). */
static inline uint64_t grow_word(uint64_t key, uint64_t den, uint64_t k) {
    return splitmix64(splitmix64(key + den) + k);
}
static inline uint32_t uniform_idx(uint32_t r, uint32_t n) {
    return (uint32_t)(((uint64_t)r * n) >> 32);
}

#define GROW_MAX_ATTEMPTS 1024

/* The source pools of one tuft: SynSrcSlices / SynSrcSliceInfo
 * (src/map/syn_src.rs:241-310,327-437). */
typedef struct {
    int8_t* ov[BM_MAX_SRC_SLICES];
    int8_t* ou[BM_MAX_SRC_SLICES];
    int on[BM_MAX_SRC_SLICES];
    int nonspatial[BM_MAX_SRC_SLICES];
    int rv[BM_MAX_SRC_SLICES], ru[BM_MAX_SRC_SLICES];
    int saturated;   /* every possible source is needed by each dendrite */
} tuft_pools;

static void free_pools(tuft_pools* Q) {
    for (int k = 0; k < BM_MAX_SRC_SLICES; k++) { free(Q->ov[k]); free(Q->ou[k]); }
}

static int make_pools(const bm_area_plan* P, const bm_tuft_plan* T, tuft_pools* Q) {
    enum { OFS_CAP = 3 * 127 * 128 + 1 };
    memset(Q, 0, sizeof *Q);
    uint64_t poss = 0;
    for (uint32_t k = 0; k < T->n_src_uniq; k++) {
        uint8_t s = T->src_uniq_slc_ids[k];
        int reach = T->src_uniq_reaches[k];
        Q->nonspatial[k] = P->slc_v_scale[s] == 0;
        if (Q->nonspatial[k]) {
            Q->rv[k] = (int)(P->slc_v_size[s] / 2);
            Q->ru[k] = (int)(P->slc_u_size[s] / 2);
            poss = (uint64_t)P->slc_v_size[s] * P->slc_u_size[s] * T->n_src;
        } else {
            Q->ov[k] = (int8_t*)malloc(OFS_CAP);
            Q->ou[k] = (int8_t*)malloc(OFS_CAP);
            Q->on[k] = bmo_gen_syn_offs(reach, P->slc_v_scale[s], P->slc_u_scale[s], Q->ov[k], Q->ou[k], OFS_CAP);
            if (Q->on[k] <= 0) { free_pools(Q); return -1; }
            Q->rv[k] = (reach * (int)P->slc_v_scale[s]) >> SLC_SCL_COEFF_L2;
            Q->ru[k] = (reach * (int)P->slc_u_scale[s]) >> SLC_SCL_COEFF_L2;
            poss = (uint64_t)Q->on[k] * T->n_src;
        }
    }
    Q->saturated = poss == T->syns_per_den;
    return 0;
}

/* One candidate source from two words of the dendrite's stream:
 * SynSrcSlices::gen_src (src/map/syn_src.rs:448-490) with its strength rule
 * (intensity = scaled reach minus offset, >> INTENSITY_REDUCTION_L2, times
 * U[-3, 3]; 0 for nonspatial slices). */
static void draw_src(const tuft_pools* Q, const bm_tuft_plan* T, uint64_t w, uint64_t w2, uint8_t* ns, int* nv,
                     int* nu, int* nstr) {
    uint32_t pi = uniform_idx((uint32_t)w, T->n_src);
    *ns = T->src_slc_ids[pi];
    uint32_t k = 0;
    while (k < T->n_src_uniq && T->src_uniq_slc_ids[k] != *ns) k++;
    if (Q->nonspatial[k]) {
        *nv = (int)uniform_idx((uint32_t)(w >> 32), (uint32_t)(2 * Q->rv[k] + 1)) - Q->rv[k];
        *nu = (int)uniform_idx((uint32_t)w2, (uint32_t)(2 * Q->ru[k] + 1)) - Q->ru[k];
        *nstr = 0;
    } else {
        uint32_t oi = uniform_idx((uint32_t)(w >> 32), (uint32_t)Q->on[k]);
        *nv = Q->ov[k][oi];
        *nu = Q->ou[k][oi];
        int inten = ((Q->rv[k] - iabs(*nv)) + (Q->ru[k] - iabs(*nu))) >> 3;
        int r = (int)uniform_idx((uint32_t)w2, 7u) - 3;
        *nstr = (int8_t)(uint8_t)(inten * r);
    }
}

/* Key of the growth stream of (area, layer, tuft). */
static inline uint64_t grow_key_of(uint64_t seed, uint32_t area, uint32_t layer, uint32_t t) {
    uint64_t key = splitmix64(seed ^ 0x67726F77ull) + (((uint64_t)area << 48) | ((uint64_t)layer << 40) | ((uint64_t)t << 32));
    return splitmix64(key);
}

/* Synapses::grow(true) (src/cortex/synapses.rs:448-501, regrow_syn :411-446):
 * every synapse draws sources from its tuft's pools; unless the pool is
 * saturated (or BM_INIT_NO_UNIQUE), a draw repeating an earlier synapse's
 * non-zero key in the same dendrite is redrawn. */
int bmo_grow(const bm_area_plan* P, uint8_t* slab, uint64_t seed, uint32_t init_flags) {
    for (uint32_t l = 0; l < P->n_layers; l++) {
        const bm_layer_plan* L = &P->layers[l];
        lview V;
        view(L, slab, &V);
        uint8_t* slc = V.b[BM_BUF_SYN_SRC_SLC_IDS];
        int8_t* vo = (int8_t*)V.b[BM_BUF_SYN_SRC_COL_V_OFFS];
        int8_t* uo = (int8_t*)V.b[BM_BUF_SYN_SRC_COL_U_OFFS];
        int8_t* str = (int8_t*)V.b[BM_BUF_SYN_STRENGTHS];
        for (uint32_t t = 0; t < L->n_tufts; t++) {
            const bm_tuft_plan* T = &L->tufts[t];
            tuft_pools Q;
            if (make_pools(P, T, &Q)) return -1;
            int unique = !(init_flags & BM_INIT_NO_UNIQUE) && !Q.saturated;
            uint64_t key = grow_key_of(seed, P->area_id, L->layer_id, t);
            int64_t n_dens = (int64_t)L->cells * T->dens_per_tft;
            int64_t cols = (int64_t)L->v_size * L->u_size;
#pragma omp parallel for schedule(static)
            for (int64_t d = 0; d < n_dens; d++) {
                uint64_t s0 = T->syn_idz + d * T->syns_per_den;
                uint64_t wk = 0;
                for (uint32_t j = 0; j < T->syns_per_den; j++) {
                    uint8_t ns = 0; int nv = 0, nu = 0; int nstr = 0;
                    for (int att = 0; att < GROW_MAX_ATTEMPTS; att++) {
                        uint64_t w = grow_word(key, d, wk++);
                        uint64_t w2 = grow_word(key, d, wk++);
                        draw_src(&Q, T, w, w2, &ns, &nv, &nu, &nstr);
                        if (!unique) break;
                        int64_t nk = (int64_t)ns * cols + (int64_t)nv * L->u_size + nu;
                        if (nk == 0) break;
                        int dup = 0;
                        for (uint32_t jj = 0; jj < j; jj++) {
                            int64_t ok = (int64_t)slc[s0 + jj] * cols + (int64_t)vo[s0 + jj] * L->u_size + uo[s0 + jj];
                            if (ok == nk) { dup = 1; break; }
                        }
                        if (!dup) break;
                    }
                    slc[s0 + j] = ns;
                    vo[s0 + j] = (int8_t)nv;
                    uo[s0 + j] = (int8_t)nu;
                    str[s0 + j] = (init_flags & BM_INIT_STRENGTH_ZERO) ? 0 : (int8_t)nstr;
                }
            }
            free_pools(&Q);
        }
    }
    return 0;
}

/* Synapses::regrow (src/cortex/synapses.rs:411-501) with SynSrcIdxCache
 * (src/map/syn_src.rs:159-211): every synapse whose strength is at or below
 * SYNAPSE_STRENGTH_FLOOR draws sources until one is accepted, in synapse
 * order within each dendrite. A source is accepted when the dendrite's source
 * set lacks its key (slice * columns + v_ofs * u_size + u_ofs), or at once
 * when the tuft's pool is saturated. The set holds every non-zero key of the
 * dendrite's current sources, plus key 0 when the dendrite's den_src_key0
 * flag says so. bismit's cache inserts the new key and, when that insert is
 * new, removes the old key: so an accepted key 0 enters the set unless the
 * synapse's old key was 0, and an old key 0 always leaves it. Growth leaves
 * every flag at 0 (the old key of every synapse is then 0). The draws come
 * from a per-(round, dendrite) stream; draws stop after GROW_MAX_ATTEMPTS,
 * keeping the last one (bismit draws until one is accepted). Sources,
 * offsets and strengths change; synapse flags do not. */
static void regrow_layer(const bm_area_plan* P, lview* V, uint64_t cyc) {
    const bm_layer_plan* L = V->L;
    uint8_t* slc = V->b[BM_BUF_SYN_SRC_SLC_IDS];
    int8_t* vo = (int8_t*)V->b[BM_BUF_SYN_SRC_COL_V_OFFS];
    int8_t* uo = (int8_t*)V->b[BM_BUF_SYN_SRC_COL_U_OFFS];
    int8_t* str = (int8_t*)V->b[BM_BUF_SYN_STRENGTHS];
    uint8_t* key0 = V->b[BM_BUF_DEN_SRC_KEY0];
    const uint64_t round = cyc / BMO_REGROW_PERIOD;
    for (uint32_t t = 0; t < L->n_tufts; t++) {
        const bm_tuft_plan* T = &L->tufts[t];
        tuft_pools Q;
        if (make_pools(P, T, &Q)) return;
        const uint64_t rkey =
            splitmix64(splitmix64(grow_key_of(P->rnd_seed, P->area_id, L->layer_id, t) ^ 0x7265677277ull) + round);
        const int64_t n_dens = (int64_t)L->cells * T->dens_per_tft;
        const int64_t cols = (int64_t)L->v_size * L->u_size;
#pragma omp parallel for schedule(static)
        for (int64_t d = 0; d < n_dens; d++) {
            const uint64_t s0 = T->syn_idz + d * T->syns_per_den;
            uint8_t* z = key0 + T->den_idz + d;
            uint64_t wk = 0;
            for (uint32_t j = 0; j < T->syns_per_den; j++) {
                if (str[s0 + j] > BMO_STRENGTH_FLOOR) continue;
                const int64_t ko = (int64_t)slc[s0 + j] * cols + (int64_t)vo[s0 + j] * L->u_size + uo[s0 + j];
                uint8_t ns = 0; int nv = 0, nu = 0, nstr = 0;
                int64_t nk = 0;
                for (int att = 0; att < GROW_MAX_ATTEMPTS; att++) {
                    uint64_t w = grow_word(rkey, d, wk++);
                    uint64_t w2 = grow_word(rkey, d, wk++);
                    draw_src(&Q, T, w, w2, &ns, &nv, &nu, &nstr);
                    nk = (int64_t)ns * cols + (int64_t)nv * L->u_size + nu;
                    if (Q.saturated) break;
                    int held;
                    if (nk == 0) {
                        held = *z != 0;
                    } else {
                        held = 0;
                        for (uint32_t jj = 0; jj < T->syns_per_den; jj++) {
                            int64_t ok = (int64_t)slc[s0 + jj] * cols + (int64_t)vo[s0 + jj] * L->u_size + uo[s0 + jj];
                            if (ok == nk) { held = 1; break; }
                        }
                    }
                    if (!held) break;
                }
                if (!Q.saturated) {
                    if (ko == 0) *z = 0;
                    else if (nk == 0) *z = 1;
                }
                slc[s0 + j] = ns;
                vo[s0 + j] = (int8_t)nv;
                uo[s0 + j] = (int8_t)nu;
                str[s0 + j] = (int8_t)nstr;
            }
        }
        free_pools(&Q);
    }
}

/* ------------------------------------------------------------ encoders --- */

static uint64_t enc_splitmix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

/* coord_hex_to_pixel, src/encode/mod.rs:52-72 (f32, as written). */
static int enc_hex_to_pixel(float v_id, float u_id, float x_size, float y_size, float hex_side, float x_ofs,
                            float y_ofs, float* xo, float* yo) {
    const float u = u_id;
    const float u_inv = 0.0f - u;
    const float v = v_id;
    const float w_inv = v + u;
    float x = w_inv * 1.5f * hex_side;
    float y = (u_inv + (w_inv / 2.0f)) * 1.73205080756f * hex_side;
    x -= x_ofs;
    y += y_ofs;
    *xo = x;
    *yo = y;
    return (y >= 0.0f && y < y_size) && (x >= 0.0f && x < x_size);
}

/* encode_2d_image (src/encode/mod.rs:66-93) with calc_offs (:36-48), whose
 * caller hands it (x_size, y_size) in the slots it names (y_size, x_size). */
void bmo_encode_image(const uint8_t* source, uint32_t x_size, uint32_t y_size, float scale_factor,
                      uint8_t* target, uint32_t v_size, uint32_t u_size) {
    const float hex_side = (float)(x_size + y_size) / (scale_factor * (float)(v_size + u_size));
    /* calc_offs(v_size, u_size, y_size := x_size, x_size := y_size, hex_side) */
    const uint32_t co_y = x_size, co_x = y_size;
    float x_ofs_inv, y_ofs_inv;
    enc_hex_to_pixel((float)(v_size >> 1), (float)(u_size >> 1), (float)co_x, (float)co_y, hex_side, 0.0f, 0.0f,
                     &x_ofs_inv, &y_ofs_inv);
    const float x_ofs = x_ofs_inv - (float)(co_x >> 1);
    const float y_ofs = (float)(co_y >> 1) - y_ofs_inv;
    for (uint32_t v = 0; v < v_size; v++)
        for (uint32_t u = 0; u < u_size; u++) {
            float x, y;
            if (enc_hex_to_pixel((float)v, (float)u, (float)x_size, (float)y_size, hex_side, x_ofs, y_ofs, &x, &y))
                target[v * u_size + u] = source[(uint32_t)y * x_size + (uint32_t)x];
        }
}

/* calc_scale, src/cmn/slice_dims.rs:201-224; -1 where the reference errs. */
static int64_t enc_calc_scale(uint32_t src_dim, uint32_t tar_dim) {
    const uint64_t src = (uint64_t)src_dim * 1024, tar = (uint64_t)tar_dim * 1024;
    if (tar == 0) return -1;
    const uint64_t incr = tar < 16 ? 1 : tar / 16;
    const uint64_t s = src / incr;
    return (s == 0 || s > 255) ? -1 : (int64_t)s;
}

/* encode_hex_mold_scaled (src/encode/write/mod.rs:190-217): -1 where the
 * scales or offsets fail, or a tile would leave the frame. */
int bmo_hex_mold(int radius, uint32_t src_v, uint32_t src_u, uint8_t* frame, uint32_t v_size, uint32_t u_size) {
    const int64_t vs = enc_calc_scale(v_size, src_v), us = enc_calc_scale(u_size, src_u);
    if (vs < 0 || us < 0) return -1;
    int8_t ov[3 * 127 * 128 + 1], ou[3 * 127 * 128 + 1];
    const int n = bmo_gen_syn_offs(radius, (uint32_t)vs, (uint32_t)us, ov, ou, 3 * 127 * 128 + 1);
    if (n < 0) return -1;
    for (int k = 0; k < n; k++) {
        const int row = ov[k] + (int)(v_size / 2), col = ou[k] + (int)(u_size / 2);
        if (row < 0 || row >= (int)v_size || col < 0 || col >= (int)u_size) return -1;
    }
    for (int k = 0; k < n; k++)
        frame[(uint32_t)((ov[k] + (int)(v_size / 2)) * (int)u_size + ou[k] + (int)(u_size / 2))] = 1;
    return n;
}

/* encode_scalar (src/encode/write/mod.rs:28-172) for frame `frame_idx` of a
 * call: clears the frame and draws the hexagon. Its random bytes (64..127)
 * come from the seeded stream (the reference's are entropy-seeded). */
int bmo_encode_scalar(float val, float lo, float hi, uint64_t seed, uint32_t frame_idx, uint8_t* frame,
                      uint32_t v_size, uint32_t u_size) {
    if (!(val >= lo && val <= hi) || v_size < 8 || u_size < 8 || !(hi > 0.0f)) return -1;
    const int vs = (int)v_size, us = (int)u_size;
    const int radius = (vs + us) / 32;
    const int extra_margin = radius + 1;
    const int margin = radius + extra_margin + 1;
    const int track_len_v = vs - (margin * 2) - 1;
    const int track_len_u = us - (margin * 2) - 1;
    const float quad_size_val = hi / 4.0f;
    const float quadrant = floorf(val / quad_size_val);
    const float quad_pos_val = val - (quad_size_val * quadrant);
#define VAL_TO_TRACT(len) ((int)((quad_pos_val / quad_size_val) * (float)(len)))
    int cv, cu;
    if (quadrant < 1.0f || quadrant >= 4.0f) {
        cv = margin;
        cu = VAL_TO_TRACT(track_len_u) + margin;
    } else if (quadrant < 2.0f) {
        cv = VAL_TO_TRACT(track_len_v) + margin;
        cu = us - margin - 1;
    } else if (quadrant < 3.0f) {
        cv = vs - margin - 1;
        cu = us - (VAL_TO_TRACT(track_len_u) + margin) - 1;
    } else {
        cv = vs - (VAL_TO_TRACT(track_len_v) + margin) - 1;
        cu = margin;
    }
#undef VAL_TO_TRACT
    const uint32_t len = v_size * u_size;
    memset(frame, 0, len);
    const uint64_t key = enc_splitmix(seed ^ 0x656E636F64657273ull);
    for (int v = -radius; v <= radius; v++) {
        const int u_z = imax(-radius, -v - radius), u_m = imin(radius, -v + radius);
        for (int u = u_z; u <= u_m; u++) {
            const int row = v + cv, col = u + cu;
            if (row < 0 || row >= vs || col < 0 || col >= us) continue;
            const uint32_t idx = (uint32_t)(row * us + col);
            frame[idx] = (uint8_t)(64 + (enc_splitmix(key + (uint64_t)frame_idx * len + idx) >> 58));
        }
    }
    return 0;
}

/* ScalarGlyphWriter (src/encode/write/scalar_glyph_writer.rs:25-151): the
 * value's tile along the track that runs around the frame's margin (clockwise
 * from the upper left), the frame cleared and the hexagon of radius
 * (v + u) / 32 around that tile set to 127. f32 arithmetic as the
 * reference's; `as u32` of the floored tile saturates (NaN to 0). */
int bmo_encode_scalar_glyph(float val, float lo, float hi, uint8_t* frame, uint32_t v_size, uint32_t u_size) {
    if (v_size < 8 || u_size < 8 || !(lo <= hi) || !(val >= lo && val <= hi)) return -1;
    const uint32_t radius = (v_size + u_size) / 32;
    const uint32_t extra_margin = radius + 1;
    const uint32_t margin = radius + extra_margin + 1;
    const uint32_t track_tiles_v = v_size - (margin * 2) - 1;
    const uint32_t track_tiles_u = u_size - (margin * 2) - 1;
    const uint32_t track_tiles_total = (track_tiles_v * 2) + (track_tiles_u * 2);
    const float track_tiles_total_f32 = (float)track_tiles_total;
    const float val_span = hi - lo;
    const uint32_t sides0 = track_tiles_u, sides1 = track_tiles_u + track_tiles_v;
    const uint32_t sides2 = (2 * track_tiles_u) + track_tiles_v, sides3 = track_tiles_total;
    const float val_pct = (val - lo) / val_span;
    const float tile_f = floorf(val_pct * track_tiles_total_f32);
    const uint32_t val_tile = !(tile_f > 0.0f) ? 0u : tile_f >= 4294967295.0f ? 0xFFFFFFFFu : (uint32_t)tile_f;
    uint32_t cv, cu;
    if (val_tile < sides0) {
        cv = margin;
        cu = margin + val_tile;
    } else if (val_tile < sides1) {
        cv = margin + (val_tile - sides0);
        cu = margin + track_tiles_u;
    } else if (val_tile < sides2) {
        cv = margin + track_tiles_v;
        cu = (margin + track_tiles_u) - (val_tile - sides1);
    } else if (val_tile < sides3) {
        cv = (margin + track_tiles_v) - (val_tile - sides2);
        cu = margin;
    } else {
        if (val_tile != track_tiles_total) return -1;
        cv = margin;
        cu = margin;
    }
    memset(frame, 0, (size_t)v_size * u_size);
    const int r = (int)radius;
    for (int v = -r; v < r + 1; v++) {
        const int u_z = imax(-r, -v - r), u_m = imin(r, -v + r);
        for (int u = u_z; u < u_m + 1; u++)
            frame[(size_t)((v + (int)cv) * (int)u_size + u + (int)cu)] = 127;
    }
    return 0;
}

/* ScalarSdrWriter::new (src/encode/write/scalar_sdr_writer.rs:96-152): the
 * waypoint count, and (when `ways` is given) the seeded waypoint table of
 * way_count x (len / 48) indices in [0, len). */
int bmo_sdr_waypoints(float lo, float hi, float way_span, uint32_t v_size, uint32_t u_size, uint64_t seed,
                      uint32_t* ways) {
    if (v_size < 8 || u_size < 8 || !(way_span > 0.0f) || !(lo <= hi)) return -1;
    const float val_span = hi - lo;
    const float val_span_norm = val_span / way_span;
    const int way_count = (int)ceilf(val_span_norm) + 1;
    const uint64_t len = (uint64_t)v_size * u_size, active = len / 48;
    if (ways) {
        const uint64_t key = enc_splitmix(seed ^ 0x7364727761797370ull);
        for (uint64_t k = 0; k < (uint64_t)way_count * active; k++)
            ways[k] = (uint32_t)(((unsigned __int128)enc_splitmix(key + k) * len) >> 64);
    }
    return way_count;
}

/* ScalarSdrWriter::encode (scalar_sdr_writer.rs:156-210). */
int bmo_sdr_encode(float val, float lo, float hi, float way_span, uint32_t way_count, const uint32_t* ways,
                   uint8_t* frame, uint32_t len) {
    if (!(val >= lo && val <= hi)) return -1;
    const uint32_t active = len / 48;
    memset(frame, 0, len);
    const float val_norm = (val - lo) / way_span;
    const float way_0 = floorf(val_norm);
    const float way_1_contrib_ratio = val_norm - way_0;
    const uint32_t way_1_contrib_count = (uint32_t)((float)active * way_1_contrib_ratio);
    const uint32_t way_0_contrib_count = active - way_1_contrib_count;
    const uint32_t way_0_idx = (uint32_t)way_0, way_1_idx = way_0_idx + 1;
    if (way_1_idx >= way_count) return -1;
    for (uint32_t k = 0; k < way_0_contrib_count; k++) frame[ways[(uint64_t)way_0_idx * active + k]] = 128;
    for (uint32_t k = way_1_contrib_count; k-- > 0;) frame[ways[(uint64_t)way_1_idx * active + k]] = 128;
    return 0;
}
