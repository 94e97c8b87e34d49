// ref_harness.cpp -- runs bismit's own OpenCL kernels on the CPU (TEST
// INFRASTRUCTURE: the reference-side checker and the reference CPU baseline).
//
// The kernel text comes verbatim from a bismit checkout (cl/bismit.cl,
// cl/syns.cl, cl/control.cl, cl/filters.cl, cl/tests.cl), prepared by prep_cl.py and compiled
// as C++ against cl_compat.hpp. This file supplies what bismit's Rust host
// supplies: the -D build options (src/cmn/mod.rs:400-442,
// src/map/area_map.rs:51-77), the NDRange of every launch and its arguments
// (the launch sites cited below), and the per-area stage order of
// CorticalArea::cycle (src/cortex/cortical_area.rs:716-789).
//
// The slice tables (the __constant arrays of cl/bismit.cl:108-114) are
// process-global here, so runs of different plans must not overlap in time.
#include <cstdint>
#include <vector>
#include <cstring>
#include <initializer_list>
#include <omp.h>

#include "../../include/bismit_b200.h"
#include "cl_compat.hpp"

// base_build_options, src/cmn/mod.rs:428-440.
#define MCOL_IS_VATIC_FLAG      1
#define CEL_PREV_CONCRETE_FLAG  128
#define CEL_BEST_IN_COL_FLAG    64
#define CEL_PREV_STPOT_FLAG     32
#define CEL_PREV_VATIC_FLAG     16
#define CEL_PREV_ACTIVE_FLAG    8
#define SYN_STPOT_FLAG          2
#define SYN_STDEP_FLAG          1
#define SYN_CONCRETE_FLAG       8
#define SYN_PREV_ACTIVE_FLAG    16
#define DEN_BASAL_PROXIMAL_FLAG 1
#define DEN_BASAL_DISTAL_FLAG   2
#define DEN_APICAL_DISTAL_FLAG  4
// gen_build_options, src/map/area_map.rs:51-61: the slice tables are filled at
// run time below, so the arrays are declared at their maximum size.
#define AXN_SLC_COUNT           256
#define SLC_SCL_COEFF_L2        4
#define AXN_SLC_IDZS            0
#define AXN_SLC_V_SIZES         0
#define AXN_SLC_U_SIZES         0
#define AXN_SLC_V_SCALES        0
#define AXN_SLC_U_SCALES        0
#define AXN_SLC_V_MIDS          0
#define AXN_SLC_U_MIDS          0

namespace clref {
#include "cl_src.inc"
}

namespace {

using clref::uchar;
using clref::uint;

static inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// The seeded per-launch value used in place of bismit's entropy-seeded
// `rng.gen::<i32>()` draws (same stream as the library and the C oracle).
static int32_t rnd_of(const bm_area_plan* P, uint32_t layer_id, uint32_t role, uint32_t tft,
                      uint64_t cycle) {
    uint64_t key = ((uint64_t)P->area_id << 40) ^ ((uint64_t)layer_id << 32) ^
                   ((uint64_t)role << 24) ^ ((uint64_t)tft << 16);
    uint64_t x = splitmix64(splitmix64(P->rnd_seed) + key);
    x = splitmix64(x + cycle);
    return (int32_t)(uint32_t)(x >> 32);
}

// Runs `kern` over an NDRange: work-groups in parallel, work-items of a group
// in order (none of the launched kernels uses barriers or local memory).
template <class F>
static int launch(size_t g0, size_t g1, size_t g2, size_t l0, size_t l1, size_t l2, F&& kern) {
    if (g0 % l0 || g1 % l1 || g2 % l2) return -1;  // CL_INVALID_WORK_GROUP_SIZE
    const long long n0 = (long long)(g0 / l0), n1 = (long long)(g1 / l1), n2 = (long long)(g2 / l2);
    const long long ng = n0 * n1 * n2;
#pragma omp parallel for schedule(static)
    for (long long g = 0; g < ng; g++) {
        clref::NDRange& r = clref::ndr;
        r.gsz[0] = g0; r.gsz[1] = g1; r.gsz[2] = g2;
        r.lsz[0] = l0; r.lsz[1] = l1; r.lsz[2] = l2;
        size_t gi0 = (size_t)(g % n0), gi1 = (size_t)((g / n0) % n1), gi2 = (size_t)(g / (n0 * n1));
        for (size_t c = 0; c < l2; c++)
            for (size_t b = 0; b < l1; b++)
                for (size_t a = 0; a < l0; a++) {
                    r.lid[0] = a; r.lid[1] = b; r.lid[2] = c;
                    r.gid[0] = gi0 * l0 + a; r.gid[1] = gi1 * l1 + b; r.gid[2] = gi2 * l2 + c;
                    kern();
                }
    }
    return 0;
}
template <class F> static int launch1(size_t g0, F&& kern) {
    size_t l0 = 1;
    for (size_t c : {256, 128, 64, 32, 16, 8, 4, 2}) if (g0 % c == 0) { l0 = c; break; }
    return launch(g0, 1, 1, l0, 1, 1, kern);
}

static void set_tables(const bm_area_plan* P) {
    for (uint32_t s = 0; s < BM_MAX_SLICES; s++) {
        bool ok = s < P->n_slices;
        clref::axn_slc_idzs[s] = ok ? P->slc_axn_idz[s] : 0;
        clref::axn_slc_v_sizes[s] = ok ? P->slc_v_size[s] : 0;
        clref::axn_slc_u_sizes[s] = ok ? P->slc_u_size[s] : 0;
        clref::axn_slc_v_scales[s] = ok ? (uchar)P->slc_v_scale[s] : 0;
        clref::axn_slc_u_scales[s] = ok ? (uchar)P->slc_u_scale[s] : 0;
        clref::axn_slc_v_mids[s] = ok ? (uchar)P->slc_v_mid[s] : 0;
        clref::axn_slc_u_mids[s] = ok ? (uchar)P->slc_u_mid[s] : 0;
    }
}

// gen_grp_centers (src/cortex/smoother.rs:11-33) with HexGroupCenters
// (src/cmn/mod.rs:809-917): six lattices, each grown from its start by the
// six moves of add_surrounds within [-r, dims + r), row-major per lattice.
static void smoother_centers(int r, int V, int U, std::vector<int>& cv, std::vector<int>& cu,
                             std::vector<size_t>& off) {
    const int l = r + 1, s = r, ls = l + s;
    const int mv[6][2] = {{-s, ls}, {l, s}, {ls, -l}, {s, -ls}, {-l, -s}, {-ls, l}};
    const int ofs = (r + 1) / 2;
    const int st[6][2] = {{0, ofs}, {-ofs, ofs}, {-ofs, 0}, {0, -ofs}, {ofs, -ofs}, {ofs, 0}};
    const int W = U + 2 * r, H = V + 2 * r;
    off.assign(7, 0);
    for (int k = 0; k < 6; k++) {
        std::vector<char> seen((size_t)W * H, 0);
        std::vector<std::pair<int, int>> todo;
        off[k] = cv.size();
        auto add = [&](int v, int u) {
            if (v < -r || u < -r || v >= V + r || u >= U + r) return;
            char& f = seen[(size_t)(v + r) * W + (u + r)];
            if (!f) { f = 1; todo.push_back({v, u}); }
        };
        add(st[k][0], st[k][1]);
        while (!todo.empty()) {
            auto c = todo.back();
            todo.pop_back();
            for (auto& m : mv) add(c.first + m[0], c.second + m[1]);
        }
        for (int v = -r; v < V + r; v++)
            for (int u = -r; u < U + r; u++)
                if (seen[(size_t)(v + r) * W + (u + r)]) { cv.push_back(v); cu.push_back(u); }
    }
    off[6] = cv.size();
}

struct Layer {
    const bm_layer_plan* L;
    uint8_t* b[BM_BUF_COUNT];
    uchar* u(int k) const { return (uchar*)b[k]; }
    char* c(int k) const { return (char*)b[k]; }
    uchar* soma() const { return L->kind == BM_LYR_SPINY_STELLATE ? u(BM_BUF_DEN_STATES) : u(BM_BUF_CEL_STATES); }
};

struct Area {
    const bm_area_plan* P;
    uchar* axns;
    Layer lyr[BM_MAX_LAYERS];
    int err = 0;
};

// Synapses::cycle, src/cortex/synapses.rs:363-387 (kernels built at :222-286).
static void syns_cycle(Area& A, Layer& Y) {
    const bm_layer_plan* L = Y.L;
    uchar* st = Y.u(BM_BUF_SYN_STATES);
    uchar* fl = Y.u(BM_BUF_SYN_FLAG_SETS);
    A.err |= launch1(L->n_syns, [&] { clref::tft_set_syn_flags(st, fl); });
    for (uint32_t t = 0; t < L->n_tufts; t++) {
        const bm_tuft_plan& T = L->tufts[t];
        uint tft_syn_idz = (uint)T.syn_idz, spt = T.syns_per_tft;
        uchar depth = (uchar)L->depth;
        if (spt % 4 == 0) {
            A.err |= launch(L->v_size, L->u_size, 1, 8, 8, 1, [&] {
                clref::layer_cycle_syns_wow_vec4(A.axns, (const clref::char4*)Y.b[BM_BUF_SYN_SRC_COL_U_OFFS],
                    (const clref::char4*)Y.b[BM_BUF_SYN_SRC_COL_V_OFFS],
                    (const clref::uchar4*)Y.b[BM_BUF_SYN_SRC_SLC_IDS], tft_syn_idz, spt, depth,
                    nullptr, nullptr, (clref::uchar4*)st);
            });
        } else {
            A.err |= launch(L->v_size, L->u_size, 1, 8, 8, 1, [&] {
                clref::layer_cycle_syns_wow(A.axns, Y.c(BM_BUF_SYN_SRC_COL_U_OFFS), Y.c(BM_BUF_SYN_SRC_COL_V_OFFS),
                    Y.u(BM_BUF_SYN_SRC_SLC_IDS), tft_syn_idz, spt, depth, nullptr, nullptr, st);
            });
        }
    }
}

// Dendrites::cycle, src/cortex/dendrites.rs:191-209 (kernel args :117-134).
static void dens_cycle(Area& A, Layer& Y, uint64_t cyc) {
    const bm_layer_plan* L = Y.L;
    syns_cycle(A, Y);
    for (uint32_t t = 0; t < L->n_tufts; t++) {
        const bm_tuft_plan& T = L->tufts[t];
        uint den_idz = (uint)T.den_idz, syn_idz = (uint)T.syn_idz, spd = T.syns_per_den, thr = T.den_threshold;
        int rnd = rnd_of(A.P, L->layer_id, BM_RND_DEN_CYCLE, t, cyc);
        A.err |= launch1((size_t)L->cells * T.dens_per_tft, [&] {
            clref::den_cycle_tft(Y.u(BM_BUF_SYN_STATES), Y.c(BM_BUF_SYN_STRENGTHS), den_idz, syn_idz, spd, thr,
                rnd, Y.u(BM_BUF_DEN_ENERGIES), Y.u(BM_BUF_DEN_ACTIVITIES), Y.u(BM_BUF_DEN_STATES_RAW), nullptr,
                nullptr, Y.u(BM_BUF_DEN_STATES));
        });
    }
}

// Control layers after the host layer's soma, in (host, exe_order) order:
// InhibitoryInterneuronNetwork::cycle (src/cortex/iinn.rs:105-127, args :38-66),
// PyrOutputter (src/cortex/pyr_outputter.rs:30-40), IntraColumnInhib
// (src/cortex/intra_column_inhib.rs:36-48).
static void controls_post(Area& A, Layer& Y, uint64_t cyc) {
    const bm_layer_plan* L = Y.L;
    uchar base = (uchar)L->base_axn_slc;
    for (uint32_t k = 0; k < L->n_ctrl; k++) {
        const bm_ctrl_plan& C = L->ctrl[k];
        if (C.kind == BM_LYR_CTRL_INHIB_BASKET) {
            if (A.P->settings & BM_SET_BYPASS_INHIB) {
                int rnd = 0;
                A.err |= launch(L->depth, L->v_size, L->u_size, 1, 1, 1, [&] {
                    clref::inhib_passthrough(Y.soma(), base, rnd, Y.u(BM_BUF_CEL_ACTIVITIES), A.axns);
                });
            } else {
                int rnd = rnd_of(A.P, C.layer_id, BM_RND_INHIB, 0, cyc);
                int radius = (int)C.field_radius;
                A.err |= launch(L->depth, L->v_size, L->u_size, 1, 8, 8, [&] {
                    clref::inhib_simple(Y.soma(), base, radius, rnd, Y.u(BM_BUF_CEL_ACTIVITIES), A.axns);
                });
            }
        } else if (C.kind == BM_LYR_CTRL_PYR_OUTPUT) {
            A.err |= launch(L->depth, L->v_size, L->u_size, 1, 1, 1, [&] {
                clref::pyr_output(Y.soma(), base, A.axns);
            });
        } else if (C.kind == BM_LYR_CTRL_INTRA_COLUMN) {
            uchar depth = (uchar)L->depth;
            A.err |= launch(L->v_size, L->u_size, 1, 1, 1, 1, [&] {
                clref::inhib_intra_column(Y.soma(), depth, base, A.axns);
            });
        } else if (C.kind == BM_LYR_CTRL_SMOOTHER) {
            // ActivitySmoother::cycle (src/cortex/smoother.rs:154-169, kernel
            // args :99-110), every cycle (its counter is never stored). The
            // centers of one lattice per launch, lattices in order: the
            // groups of a lattice are disjoint, so its work-items may run in
            // any order.
            int radius = (int)C.field_radius;
            uchar depth = (uchar)L->depth;
            uint v_size = L->v_size, u_size = L->u_size;
            std::vector<int> cv, cu;
            std::vector<size_t> off;
            smoother_centers(radius, (int)v_size, (int)u_size, cv, cu, off);
            for (int k = 0; k < 6; k++) {
                const size_t n = off[k + 1] - off[k];
                if (!n) continue;
                const int* pv = cv.data() + off[k];
                const int* pu = cu.data() + off[k];
                A.err |= launch(n, 1, 1, 1, 1, 1, [&] {
                    clref::smooth_activity(pv, pu, v_size, u_size, radius, depth, Y.u(BM_BUF_CEL_ACTIVITIES),
                                           Y.u(BM_BUF_CEL_ENERGIES));
                });
            }
        }
    }
}

// Tufts::learn, src/cortex/tufts.rs:288-333 (kernel args :151-208).
static void tufts_learn(Area& A, Layer& Y, uint64_t cyc) {
    const bm_layer_plan* L = Y.L;
    if (A.P->settings & (BM_SET_DISABLE_LEARNING | BM_SET_DISABLE_PYRS)) return;
    for (uint32_t t = 0; t < L->n_tufts; t++) {
        const bm_tuft_plan& T = L->tufts[t];
        if (T.den_kind != BM_DEN_DISTAL) continue;
        if (L->cells % 64) { A.err |= -2; return; }  // CorticalDims::per_subgrp panics
        uint cel_idz = (uint)T.cel_idz, den_idz = (uint)T.den_idz, syn_idz = (uint)T.syn_idz;
        uint dpt = T.dens_per_tft, spd = T.syns_per_den, spt = T.syns_per_tft;
        uint cpg = L->cells / 64, axn_idz = L->axn_idz;
        int rnd = rnd_of(A.P, L->layer_id, BM_RND_TFT_DST_MTP, t, cyc);
        A.err |= launch(64, 1, 1, 1, 1, 1, [&] {
            clref::tft_dst_mtp(A.axns, Y.u(BM_BUF_CEL_STATES), Y.u(BM_BUF_TFT_PREV_BEST_DEN_IDS),
                Y.u(BM_BUF_TFT_PREV_BEST_DEN_STATES_RAW), Y.u(BM_BUF_DEN_STATES), Y.u(BM_BUF_SYN_STATES),
                cel_idz, den_idz, syn_idz, dpt, spd, spt, cpg, axn_idz, 0, 5, rnd,
                Y.u(BM_BUF_SYN_FLAG_SETS), Y.u(BM_BUF_CEL_FLAG_SETS), nullptr, nullptr,
                Y.c(BM_BUF_SYN_STRENGTHS));
        });
    }
}

// SpinyStellateLayer::learn, src/cortex/spiny_stellates.rs:256-266 (args :98-112).
static void ssc_learn(Area& A, Layer& Y, uint64_t cyc) {
    const bm_layer_plan* L = Y.L;
    if (A.P->settings & (BM_SET_DISABLE_LEARNING | BM_SET_DISABLE_SSCS)) return;
    uint axn_idz = L->axn_idz, spt = L->tufts[0].syns_per_tft;
    uint rnd = (uint)rnd_of(A.P, L->layer_id, BM_RND_SSC_MTP, 0, cyc);
    A.err |= launch(1, L->cells, 1, 1, 1, 1, [&] {
        clref::ssc_mtp_simple(A.axns, Y.u(BM_BUF_SYN_STATES), axn_idz, spt, rnd, Y.c(BM_BUF_SYN_STRENGTHS));
    });
}

static void layer_cycle(Area& A, Layer& Y, uint64_t cyc) {
    const bm_layer_plan* L = Y.L;
    if (L->kind == BM_LYR_SPINY_STELLATE) {
        // SpinyStellateLayer::cycle, src/cortex/spiny_stellates.rs:220-252.
        dens_cycle(A, Y, cyc);
        A.err |= launch(L->depth, L->v_size, L->u_size, 1, 1, 1, [&] {
            clref::ssc_cycle(Y.u(BM_BUF_CEL_ENERGIES), Y.u(BM_BUF_DEN_STATES));
        });
        controls_post(A, Y, cyc);
    } else {
        // PyramidalLayer::cycle, src/cortex/pyramidals.rs:297-335; Tufts::cycle
        // src/cortex/tufts.rs:335-358 (tft_cycle args :107-127); pyr_cycle args
        // src/cortex/pyramidals.rs:148-165.
        dens_cycle(A, Y, cyc);
        for (uint32_t t = 0; t < L->n_tufts; t++) {
            const bm_tuft_plan& T = L->tufts[t];
            uint cel_idz = (uint)T.cel_idz, den_idz = (uint)T.den_idz, dpt = T.dens_per_tft;
            uchar mad = (uchar)T.max_active_dens_l2;
            A.err |= launch1(L->cells, [&] {
                clref::tft_cycle(Y.u(BM_BUF_DEN_STATES_RAW), Y.u(BM_BUF_DEN_STATES), cel_idz, den_idz, dpt, mad,
                    Y.u(BM_BUF_TFT_PREV_BEST_DEN_IDS), Y.u(BM_BUF_TFT_PREV_BEST_DEN_STATES_RAW),
                    Y.u(BM_BUF_TFT_PREV_BEST_DEN_STATES), Y.u(BM_BUF_TFT_PREV_STATES),
                    Y.u(BM_BUF_TFT_BEST_DEN_IDS), Y.u(BM_BUF_TFT_BEST_DEN_STATES_RAW),
                    Y.u(BM_BUF_TFT_BEST_DEN_STATES), nullptr, nullptr, Y.u(BM_BUF_TFT_STATES));
            });
        }
        uchar tft_count = (uchar)L->n_tufts, fl = (uchar)L->enabled_tft_flags;
        uchar prx = (uchar)L->bsl_prx_tft_id, dst = (uchar)L->bsl_dst_tft_id, apc = (uchar)L->apc_dst_tft_id;
        A.err |= launch1(L->cells, [&] {
            clref::pyr_cycle(Y.u(BM_BUF_TFT_BEST_DEN_STATES_RAW), Y.u(BM_BUF_TFT_STATES), tft_count, fl, prx,
                dst, apc, nullptr, nullptr, Y.u(BM_BUF_CEL_STATES));
        });
        controls_post(A, Y, cyc);
        tufts_learn(A, Y, cyc);
    }
}

static void layer_learn(Area& A, Layer& Y, uint64_t cyc) {
    if (Y.L->kind == BM_LYR_SPINY_STELLATE) ssc_learn(A, Y, cyc);
    else tufts_learn(A, Y, cyc);
}

static bool filters_run(const bm_area_plan* P) {
    return P->n_filter_chains && !(P->settings & BM_SET_BYPASS_FILTERS);
}

// One frame of input 0: a source with a running filter chain goes to the
// chain's first buffer (SensoryFilter::write, src/cortex/sensory_filter.rs:
// 122-155), the rest to the input's axons (AxonSpace::intake,
// src/cortex/axon_space.rs:510-560).
static void intake(const bm_area_plan* P, uint8_t* slab, const uint8_t* frame) {
    const bm_io_plan& io = P->inputs[0];
    uint8_t* axns = slab + P->axon_off + io.axn_idz;
    for (uint32_t b = 0; b < io.len; b++) {
        uint8_t* dst = axns + b;
        for (uint32_t k = 0; filters_run(P) && k < P->n_filter_chains; k++) {
            const bm_filter_chain_plan& c = P->filter_chains[k];
            const uint32_t c0 = c.frame_off, c1 = c0 + c.depth * c.v_size * c.u_size;
            if (c.input == 0 && b >= c0 && b < c1) dst = slab + c.buf_off[0] + (b - c0);
        }
        *dst = frame[b];
    }
}

// SensoryFilter::cycle of every filter of each chain in order: the
// (depth, v, u) NDRange in 1 x 8 x 8 work-groups, arguments (input buffer,
// output slice base, output buffer) as SensoryFilter::new binds them
// (src/cortex/sensory_filter.rs:47-54; the last filter's output is the axon
// space at the target slices, an inner one's the next filter's buffer from
// slice 0, src/cortex/axon_space.rs:353-365).
static void run_filters(Area& A, uint8_t* slab) {
    if (!filters_run(A.P)) return;
    for (uint32_t k = 0; k < A.P->n_filter_chains; k++) {
        const bm_filter_chain_plan& c = A.P->filter_chains[k];
        for (uint32_t f = 0; f < c.n_filters; f++) {
            const bool last = f + 1 == c.n_filters;
            const uchar* in = slab + c.buf_off[f];
            uchar* out = last ? A.axns : slab + c.buf_off[f + 1];
            const uchar base = (uchar)(last ? c.tar_slc : 0);
            A.err |= launch(c.depth, c.v_size, c.u_size, 1, 8, 8, [&] { clref::retina(in, base, out); });
        }
    }
}

}  // namespace

extern "C" {

// Runs n_cycles cycles with the reference kernels; same contract as bmo_run.
int bmr_run(const bm_area_plan* P, uint8_t* slab, const uint8_t* frames, uint64_t frame_len,
            uint32_t n_cycles, uint64_t start_cycle, int n_threads) {
    if (n_threads > 0) omp_set_num_threads(n_threads);
    if (frames && (P->n_inputs == 0 || frame_len != P->inputs[0].len)) return -1;
    set_tables(P);
    Area A;
    A.P = P;
    A.axns = slab + P->axon_off;
    for (uint32_t l = 0; l < P->n_layers; l++) {
        A.lyr[l].L = &P->layers[l];
        for (int k = 0; k < BM_BUF_COUNT; k++)
            A.lyr[l].b[k] = P->layers[l].buf_off[k] == UINT64_MAX ? nullptr : slab + P->layers[l].buf_off[k];
    }
    for (uint32_t k = 0; k < n_cycles; k++) {
        uint64_t cyc = start_cycle + k;
        if (frames) intake(P, slab, frames + (uint64_t)k * frame_len);
        run_filters(A, slab);
        // CorticalArea::cycle, src/cortex/cortical_area.rs:716-789.
        if (!(P->settings & BM_SET_DISABLE_SSCS)) {
            for (uint32_t i = 0; i < P->n_cycle_order; i++) {
                Layer& Y = A.lyr[P->cycle_order[i]];
                if (Y.L->tags & BM_TAG_SPATIAL) layer_cycle(A, Y, cyc);
            }
            for (uint32_t i = 0; i < P->n_cycle_order; i++) {
                Layer& Y = A.lyr[P->cycle_order[i]];
                if (Y.L->tags & BM_TAG_SPATIAL) layer_learn(A, Y, cyc);
            }
        }
        if (!(P->settings & BM_SET_DISABLE_PYRS)) {
            for (uint32_t i = 0; i < P->n_cycle_order; i++) {
                Layer& Y = A.lyr[P->cycle_order[i]];
                if (!(Y.L->tags & BM_TAG_SPATIAL)) layer_cycle(A, Y, cyc);
            }
        }
        if (A.err) return -3;
    }
    return 0;
}

// The `kernels` test of src/tests/kernels.rs:21-91: runs test_axn_idxs_scl and
// test_axn_idxs_vec4 (cl/tests.cl:15-85) over a (depth, v, u) grid with the
// given i8 offsets and writes both index arrays.
int bmr_test_axn_idxs(const bm_area_plan* P, uint32_t depth, uint32_t v_size, uint32_t u_size,
                      const int8_t* v_offs, const int8_t* u_offs, uint32_t* outs_scl, uint32_t* outs_v4) {
    if (u_size % 4) return -1;
    set_tables(P);
    int err = launch(depth, v_size, u_size, 1, 1, 1, [&] {
        clref::test_axn_idxs_scl((const char*)v_offs, (const char*)u_offs, outs_scl);
    });
    err |= launch(depth, v_size, u_size / 4, 1, 1, 1, [&] {
        clref::test_axn_idxs_vec4((const clref::char4*)v_offs, (const clref::char4*)u_offs, (clref::uint4*)outs_v4);
    });
    return err;
}

}  // extern "C"
