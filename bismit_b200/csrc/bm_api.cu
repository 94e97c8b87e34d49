// bm_api.cu -- the C ABI (include/bismit_b200.h): contexts, areas, the cycle
// scheduler and buffer I/O. The stage order is CorticalArea::cycle
// (src/cortex/cortical_area.rs:716-789) with the layer cycles of
// SpinyStellateLayer::cycle (src/cortex/spiny_stellates.rs:220-252) and
// PyramidalLayer::cycle (src/cortex/pyramidals.rs:297-335).
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "bm_area.h"
#include "bm_layout.h"

using namespace bm;

namespace {

thread_local char g_err[1024];

}  // namespace

int bm::set_err(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

int bm::cuda_err(cudaError_t e, const char* what) {
    return set_err(e == cudaErrorMemoryAllocation ? BM_ERR_OOM : BM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

namespace {

#define CU(call)                                                   \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return cuda_err(e_, #call);         \
    } while (0)

}  // namespace

// ------------------------------------------------------- stage program ---
namespace {

void push_controls(const bm_area_s* A, uint32_t i, std::vector<Step>& out) {
    const bm_layer_plan& L = A->plan.layers[i];
    for (uint32_t k = 0; k < L.n_ctrl; k++) {
        const uint32_t kind = L.ctrl[k].kind;
        uint8_t st;
        if (kind == BM_LYR_CTRL_INHIB_BASKET)
            st = (A->plan.settings & BM_SET_BYPASS_INHIB) ? ST_INHIB_PASS : ST_INHIB_SIMPLE;
        else if (kind == BM_LYR_CTRL_PYR_OUTPUT)
            st = ST_PYR_OUTPUT;
        else if (kind == BM_LYR_CTRL_INTRA_COLUMN)
            st = ST_INTRA_COL;
        else if (kind == BM_LYR_CTRL_SMOOTHER)
            st = ST_SMOOTH;
        else
            continue;
        out.push_back({st, (uint8_t)i, (uint8_t)k, 0});
    }
}

void push_pyr_learn(const bm_area_s* A, uint32_t i, std::vector<Step>& out) {
    const bm_layer_plan& L = A->plan.layers[i];
    if (A->plan.settings & (BM_SET_DISABLE_LEARNING | BM_SET_DISABLE_PYRS)) return;
    for (uint32_t t = 0; t < L.n_tufts; t++)
        if (L.tufts[t].den_kind == BM_DEN_DISTAL) out.push_back({ST_DST_MTP, (uint8_t)i, (uint8_t)t, 0});
}

// SpinyStellateLayer::cycle (src/cortex/spiny_stellates.rs:220-252) and
// PyramidalLayer::cycle (src/cortex/pyramidals.rs:297-335, learning included).
void push_layer_cycle(const bm_area_s* A, uint32_t i, std::vector<Step>& out) {
    const bm_layer_plan& L = A->plan.layers[i];
    if (A->exec_path == BM_PATH_PLAIN)
        out.push_back({ST_TUFTS_PLAIN, (uint8_t)i, 0, 0});
    else
        for (uint32_t t = 0; t < L.n_tufts; t++) out.push_back({ST_TUFT, (uint8_t)i, (uint8_t)t, 0});
    if (L.kind == BM_LYR_SPINY_STELLATE) {
        out.push_back({ST_SSC_CYCLE, (uint8_t)i, 0, 0});
        push_controls(A, i, out);
    } else {
        out.push_back({ST_PYR_CYCLE, (uint8_t)i, 0, 0});
        push_controls(A, i, out);
        push_pyr_learn(A, i, out);
    }
}

void push_layer_learn(const bm_area_s* A, uint32_t i, std::vector<Step>& out) {
    const bm_layer_plan& L = A->plan.layers[i];
    if (L.kind == BM_LYR_SPINY_STELLATE) {
        if (!(A->plan.settings & (BM_SET_DISABLE_LEARNING | BM_SET_DISABLE_SSCS)))
            out.push_back({ST_SSC_MTP, (uint8_t)i, 0, 0});
    } else {
        push_pyr_learn(A, i, out);
    }
}

// Slices of data layer i are plain: unscaled, unshifted and laid out back to
// back from the layer's first axon, so the axon a control writes for cell c
// is axn_idz + c.
bool layer_plain(const bm_area_plan& P, uint32_t i) {
    const bm_layer_plan& L = P.layers[i];
    const uint32_t cols = L.v_size * L.u_size;
    for (uint32_t s = 0; s < L.depth; s++) {
        const uint32_t k = L.base_axn_slc + s;
        if (k >= P.n_slices) return false;
        if (P.slc_v_scale[k] != 16 || P.slc_u_scale[k] != 16 || P.slc_v_mid[k] || P.slc_u_mid[k]) return false;
        if (P.slc_v_size[k] != L.v_size || P.slc_u_size[k] != L.u_size) return false;
        if (P.slc_axn_idz[k] != L.axn_idz + s * cols) return false;
    }
    return true;
}

// Fused forms of adjacent steps whose later stages only read what the earlier
// ones wrote for the same cell (bm_items.cuh).
void fuse_steps(const bm_area_s* A, std::vector<Step>& v, bool fold_cell_tufts) {
    const bm_area_plan& P = A->plan;
    std::vector<Step> out;
    for (size_t k = 0; k < v.size(); k++) {
        const Step& s = v[k];
        // A spiny stellate tuft whose cells have one dendrite, taken by the
        // fused kernel, also runs the ssc_cycle that follows it (arg 1): the
        // soma is that dendrite's state, known in the same launch.
        if (s.kind == ST_TUFT && k + 1 < v.size() && v[k + 1].kind == ST_SSC_CYCLE && v[k + 1].layer == s.layer &&
            P.layers[s.layer].kind == BM_LYR_SPINY_STELLATE && P.layers[s.layer].n_tufts == 1 &&
            P.layers[s.layer].tufts[0].dens_per_tft == 1 && A->fused.t[s.layer][s.idx].ok) {
            out.push_back({ST_TUFT, s.layer, s.idx, 1});
            k++;
            continue;
        }
        if (s.kind == ST_INHIB_SIMPLE && layer_plain(P, s.layer) &&
            P.layers[s.layer].kind == BM_LYR_SPINY_STELLATE) {
            const bool learn = k + 1 < v.size() && v[k + 1].kind == ST_SSC_MTP && v[k + 1].layer == s.layer;
            out.push_back({ST_INHIB_MTP, s.layer, s.idx, (uint8_t)learn});
            if (learn) k++;
            continue;
        }
        if (s.kind == ST_PYR_CYCLE && layer_plain(P, s.layer)) {
            const bm_layer_plan& L = P.layers[s.layer];
            size_t j = k + 1;
            uint8_t ctrl = 0xFF;
            if (j < v.size() && v[j].layer == s.layer && (v[j].kind == ST_INTRA_COL || v[j].kind == ST_PYR_OUTPUT)) {
                ctrl = v[j].idx;
                j++;
            }
            // Every distal tuft's learning, in tuft order, or none.
            size_t m = j;
            bool all = true;
            uint32_t n_dst = 0;
            for (uint32_t t = 0; t < L.n_tufts; t++) {
                if (L.tufts[t].den_kind != BM_DEN_DISTAL) continue;
                n_dst++;
                if (m < v.size() && v[m].kind == ST_DST_MTP && v[m].layer == s.layer && v[m].idx == t) m++;
                else all = false;
            }
            const bool learn = n_dst > 0 && all;
            if (learn || m == j) {
                // The layer's tuft steps that run per cell (tufts the fused
                // kernel does not take) come right before its soma step with
                // only other tuft steps of the layer in between, which write
                // no axon: they fold into the tail, each cell's four stages
                // ahead of its soma.
                uint8_t tufts = 0;
                for (size_t q = out.size(); q > 0 && fold_cell_tufts; q--) {
                    const Step& o = out[q - 1];
                    if (o.kind != ST_TUFT || o.layer != s.layer) break;
                    if (!A->fused.t[s.layer][o.idx].ok && o.idx < 8) tufts |= (uint8_t)(1u << o.idx);
                }
                if (tufts)
                    out.erase(std::remove_if(out.begin(), out.end(),
                                             [&](const Step& o) {
                                                 return o.kind == ST_TUFT && o.layer == s.layer &&
                                                        ((tufts >> o.idx) & 1);
                                             }),
                              out.end());
                Step tail{ST_PYR_TAIL, s.layer, ctrl, (uint8_t)learn};
                tail.tufts = tufts;
                out.push_back(tail);
                k = (learn ? m : j) - 1;
                continue;
            }
        }
        out.push_back(s);
    }
    v.swap(out);
}

}  // namespace

// CorticalArea::cycle, src/cortex/cortical_area.rs:716-789 (intake happens
// before the cycle; output is read on demand), with CorticalArea::regrow
// (src/cortex/cortical_area.rs:792-806) as a step of every cycle that acts on
// the cycles its counter fires.
uint64_t bm::cell_tuft_cells(const bm_area_s* A) {
    const bm_area_plan& P = A->plan;
    uint64_t n = 0;
    for (uint32_t i = 0; i < P.n_layers; i++) {
        if (P.layers[i].kind != BM_LYR_PYRAMIDAL) continue;
        bool cell_tuft = false;
        for (uint32_t t = 0; t < P.layers[i].n_tufts; t++) cell_tuft |= !A->fused.t[i][t].ok;
        if (cell_tuft) n += P.layers[i].cells;
    }
    return n;
}

void bm::area_steps(const bm_area_s* A, std::vector<Step>& out, bool fold_cell_tufts) {
    const bm_area_plan& P = A->plan;
    out.clear();
    // AxonSpace::intake (src/cortex/axon_space.rs:510-525): each filtered
    // input's chain runs before the layers.
    if (filters_run(P))
        for (uint32_t c = 0; c < P.n_filter_chains; c++) out.push_back({ST_FILTER, 0, (uint8_t)c, 0});
    if (!(P.settings & BM_SET_DISABLE_SSCS)) {
        for (uint32_t k = 0; k < P.n_cycle_order; k++)
            if (P.layers[P.cycle_order[k]].tags & BM_TAG_SPATIAL) push_layer_cycle(A, P.cycle_order[k], out);
        for (uint32_t k = 0; k < P.n_cycle_order; k++)
            if (P.layers[P.cycle_order[k]].tags & BM_TAG_SPATIAL) push_layer_learn(A, P.cycle_order[k], out);
    }
    if (!(P.settings & BM_SET_DISABLE_PYRS)) {
        for (uint32_t k = 0; k < P.n_cycle_order; k++)
            if (!(P.layers[P.cycle_order[k]].tags & BM_TAG_SPATIAL)) push_layer_cycle(A, P.cycle_order[k], out);
    }
    if (A->regrow_blocks) out.push_back({ST_REGROW, 0, 0, 0});
    out.push_back({ST_CYCLE_END, 0, 0, 0});
    if (A->exec_path == BM_PATH_FUSED) fuse_steps(A, out, fold_cell_tufts);
}

// Synapse flags, synapse cycle, dendrite cycle and (pyramidal) tuft cycle: the
// plain form launches them as bismit does (flags over the whole layer, then
// each stage per tuft); the fused form takes each tuft on its own, one fused
// launch where the tuft qualifies, else that tuft's four stages. The stages of
// different tufts touch disjoint buffers, so both orders give the same bytes.
void bm::exec_step(bm_area_s* A, const Step& st, cudaStream_t s, bool end_cycle) {
    const uint32_t i = st.layer, x = st.idx;
    const bm_layer_plan& L = A->plan.layers[i];
    const DevLayer& D = A->dl[i];
    const bool pyr = L.kind == BM_LYR_PYRAMIDAL;
    // Launches on the area's own stream are counted (and timed when profiling);
    // a batch passes its own stream and does its own counting.
    const bool front = A->front && s == A->front;
    const bool own = s == A->stream() || (A->side && s == A->side) || front;
    // Launches on the front stream may run ahead of the area's counter: they
    // take the number of the cycle being enqueued from the host.
    const int64_t host_cycle = front ? (int64_t)A->host_cycle : -1;
    auto run = [&](int kind, auto&& f) {
        if (own) A->run(kind, f);
        else f();
    };
    switch (st.kind) {
    case ST_TUFT:
        if (A->fused.t[i][x].ok) {
            run(K_FUSED_TUFT,
                [&] { launch_fused_tuft(A->fused, A->axns(), A->slices, D, i, x, A->ctl, s, (st.arg & 1) != 0, host_cycle); });
        } else {
            run(K_TUFT_CELLS, [&] { launch_tuft_cells(A->axns(), A->slices, D, x, A->ctl, s); });
        }
        break;
    case ST_INHIB_MTP:
        run(K_INHIB_MTP, [&] {
            launch_inhib_mtp(A->axns(), A->slices, D, (int)L.ctrl[x].field_radius, A->inhib_key[i][x], st.arg != 0,
                             A->ctl, s, host_cycle);
        });
        break;
    case ST_PYR_TAIL: {
        const int ctrl = x == 0xFF ? 0 : (L.ctrl[x].kind == BM_LYR_CTRL_INTRA_COLUMN ? 1 : 2);
        run(K_PYR_TAIL,
            [&] { launch_pyr_tail(A->axns(), A->slices, D, ctrl, st.arg != 0, A->ctl, s, st.tufts, end_cycle); });
        break;
    }
    case ST_TUFTS_PLAIN:
        run(K_SYN_FLAGS, [&] { launch_set_syn_flags(D, s); });
        for (uint32_t t = 0; t < L.n_tufts; t++)
            run(K_SYN_CYCLE, [&] { launch_syn_cycle_plain(A->axns(), A->slices, D, t, s); });
        for (uint32_t t = 0; t < L.n_tufts; t++) run(K_DEN_CYCLE, [&] { launch_den_cycle_plain(D, t, A->ctl, s); });
        if (pyr)
            for (uint32_t t = 0; t < L.n_tufts; t++) run(K_TFT_CYCLE, [&] { launch_tft_cycle_plain(D, t, s); });
        break;
    case ST_SSC_CYCLE: run(K_SSC_CYCLE, [&] { launch_ssc_cycle(D, s); }); break;
    case ST_INHIB_SIMPLE:
        run(K_INHIB_SIMPLE, [&] {
            launch_inhib_simple(A->axns(), A->slices, D, (int)L.ctrl[x].field_radius, A->inhib_key[i][x], A->ctl, s);
        });
        break;
    case ST_INHIB_PASS: run(K_INHIB_PASS, [&] { launch_inhib_passthrough(A->axns(), A->slices, D, s); }); break;
    case ST_PYR_OUTPUT: run(K_PYR_OUTPUT, [&] { launch_pyr_output(A->axns(), A->slices, D, s); }); break;
    case ST_INTRA_COL: run(K_INTRA_COL, [&] { launch_inhib_intra_column_plain(A->axns(), A->slices, D, s); }); break;
    case ST_PYR_CYCLE: run(K_PYR_CYCLE, [&] { launch_pyr_cycle_plain(D, s); }); break;
    case ST_DST_MTP: run(K_TFT_DST_MTP, [&] { launch_tft_dst_mtp_plain(A->axns(), D, x, A->ctl, s); }); break;
    case ST_SSC_MTP: run(K_SSC_MTP, [&] { launch_ssc_mtp_plain(A->axns(), D, A->ctl, s); }); break;
    case ST_REGROW:
        // Only the area's own cycles come here, enqueued as they run, with
        // host_cycle the number of the cycle being enqueued: the launch is
        // left out on the cycles it would return at once (graph-replayed
        // batches launch it every cycle and let the device decide).
        if (A->host_cycle % kRegrowPeriod != kRegrowPeriod - 1) break;
        run(K_REGROW, [&] { launch_regrow(A->d_regrow, (uint32_t)A->regrow.size(), A->regrow_blocks, s); });
        break;
    case ST_SMOOTH: {
        // The six lattices in order (the reference runs them as one racing
        // launch; this is one of the orders it can produce).
        const uint32_t* off = A->center_off[i][x];
        for (int k = 0; k < 6; k++)
            run(K_SMOOTH, [&] {
                launch_smooth(D, A->d_centers[i][x] + off[k], off[k + 1] - off[k], (int32_t)L.ctrl[x].field_radius, s);
            });
        break;
    }
    case ST_FILTER: {
        // SensoryFilter::cycle (src/cortex/sensory_filter.rs:157-168) of each
        // filter in order: filter k reads its own buffer and writes the next
        // one's (slice offsets from slice 0, cl/filters.cl:45-47), the last
        // the target slices.
        const bm_filter_chain_plan& c = A->plan.filter_chains[x];
        for (uint32_t f = 0; f < c.n_filters; f++) {
            const bool last = f + 1 == c.n_filters;
            uint8_t* out = last ? A->axns() : A->slab + c.buf_off[f + 1];
            run(K_RETINA, [&] {
                launch_retina(A->slab + c.buf_off[f], out, A->slices, last ? c.tar_slc : 0, c.depth, c.v_size,
                              c.u_size, s);
            });
        }
        break;
    }
    case ST_CYCLE_END: run(K_CYCLE_END, [&] { launch_cycle_end(A->ctl, s); }); break;
    default: break;
    }
}

namespace {

void layer_axons(const bm_area_plan& P, uint32_t i, std::bitset<BM_MAX_SLICES>& out) {
    const bm_layer_plan& L = P.layers[i];
    for (uint32_t k = 0; k < L.depth && L.base_axn_slc + k < BM_MAX_SLICES; k++) out.set(L.base_axn_slc + k);
}

void tuft_sources(const bm_area_plan& P, uint32_t i, uint32_t t, std::bitset<BM_MAX_SLICES>& out) {
    const bm_tuft_plan& T = P.layers[i].tufts[t];
    for (uint32_t k = 0; k < T.n_src_uniq; k++) out.set(T.src_uniq_slc_ids[k]);
}

uint64_t tuft_bit(uint32_t i, uint32_t t) { return 1ull << (i * BM_MAX_TUFTS + t); }
uint64_t layer_tufts(const bm_area_plan& P, uint32_t i) {
    uint64_t m = 0;
    for (uint32_t t = 0; t < P.layers[i].n_tufts; t++) m |= tuft_bit(i, t);
    return m;
}

}  // namespace

// Reads and writes of each step kind (the item bodies in bm_items.cuh, the
// fused kernels in bm_fused.cu); learning steps are taken to read every axon.
bm::StepAccess bm::step_access(const bm_area_s* A, const Step& st, int t) {
    const bm_area_plan& P = A->plan;
    const uint32_t i = st.layer;
    StepAccess a;
    switch (st.kind) {
    case ST_TUFT: {
        const uint32_t tt = t >= 0 ? (uint32_t)t : st.idx;
        if ((A->foreign_src[i] >> tt) & 1) a.ax_r.set();   // sources anywhere: any slice
        else tuft_sources(P, i, tt, a.ax_r);
        a.tf_r = a.tf_w = tuft_bit(i, tt);
        if (st.arg & 1) a.ce_r = a.ce_w = 1u << i;          // with the folded ssc_cycle
        break;
    }
    case ST_TUFTS_PLAIN:
        if (A->foreign_src[i]) a.ax_r.set();
        else
            for (uint32_t k = 0; k < P.layers[i].n_tufts; k++) tuft_sources(P, i, k, a.ax_r);
        a.tf_r = a.tf_w = layer_tufts(P, i);
        break;
    case ST_SSC_CYCLE:
    case ST_PYR_CYCLE:
        a.tf_r = layer_tufts(P, i);
        a.ce_r = a.ce_w = 1u << i;
        break;
    case ST_INHIB_SIMPLE:
    case ST_INHIB_PASS:
        a.ce_r = a.ce_w = 1u << i;
        layer_axons(P, i, a.ax_w);
        break;
    case ST_INHIB_MTP:
    case ST_SSC_MTP:
        a.ce_r = a.ce_w = 1u << i;
        layer_axons(P, i, a.ax_w);
        a.ax_r = a.ax_w;
        a.tf_r = a.tf_w = layer_tufts(P, i);
        break;
    case ST_PYR_OUTPUT:
    case ST_INTRA_COL:
        a.ce_r = 1u << i;
        layer_axons(P, i, a.ax_w);
        break;
    case ST_SMOOTH:
        a.ce_r = a.ce_w = 1u << i;
        break;
    case ST_FILTER: {
        // Reads the chain's own buffers, which nothing else in a cycle touches.
        const bm_filter_chain_plan& c = P.filter_chains[st.idx];
        for (uint32_t k = 0; k < c.depth; k++) a.ax_w.set(c.tar_slc + k);
        break;
    }
    case ST_DST_MTP:
    case ST_PYR_TAIL:
        // The layer's own axons (soma output, learning's activity test), and
        // the sources of the per-cell tufts folded into the tail.
        layer_axons(P, i, a.ax_r);
        for (uint32_t t = 0; t < P.layers[i].n_tufts && st.kind == ST_PYR_TAIL; t++)
            if ((st.tufts >> t) & 1) {
                if ((A->foreign_src[i] >> t) & 1) a.ax_r.set();
                else tuft_sources(P, i, t, a.ax_r);
            }
        layer_axons(P, i, a.ax_w);
        a.tf_r = a.tf_w = layer_tufts(P, i);
        a.ce_r = a.ce_w = 1u << i;
        break;
    default:
        a.all = true;
        break;
    }
    return a;
}

// A tuft step whose accesses conflict with no earlier step left on the main
// stream runs on the side stream (side steps keep their order there); a main
// step waits for each earlier side step it conflicts with, and the cycle's end
// for all of them. Concurrent steps touch disjoint bytes, so the result is
// the sequential program's.
// Records which tufts of layer i may hold source slice ids outside their
// pools after the caller wrote slice ids [b, e) of the layer (`data`, or
// null when the bytes are not known here). With `exact` the write covered the
// whole layer and replaces the record; else it can only add to it.
void bm::note_sources(bm_area_s* A, uint32_t i, uint64_t b, uint64_t e, const uint8_t* data, bool exact) {
    const bm_layer_plan& L = A->plan.layers[i];
    uint8_t mark = 0;
    for (uint32_t t = 0; t < L.n_tufts; t++) {
        const bm_tuft_plan& T = L.tufts[t];
        const uint64_t lo = std::max<uint64_t>(b, T.syn_idz);
        const uint64_t hi = std::min<uint64_t>(e, T.syn_idz + (uint64_t)L.cells * T.syns_per_tft);
        if (lo >= hi) continue;
        if (!data) {
            mark |= (uint8_t)(1u << t);
            continue;
        }
        bool pool[256] = {};
        for (uint32_t k = 0; k < T.n_src_uniq; k++) pool[T.src_uniq_slc_ids[k]] = true;
        for (uint64_t x = lo; x < hi; x++)
            if (!pool[data[x - b]]) {
                mark |= (uint8_t)(1u << t);
                break;
            }
    }
    const uint8_t next = exact ? mark : (uint8_t)(A->foreign_src[i] | mark);
    if (next == A->foreign_src[i]) return;
    A->foreign_src[i] = next;
    A->access_version++;
    schedule_area(A);
}

namespace {

// A step the front stream can take: a spatial layer's fused tuft (with its
// folded soma step) or its inhibition with learning; their kernels take the
// cycle number from the host.
bool front_step_ok(const bm_area_s* A, const Step& st) {
    const bm_area_plan& P = A->plan;
    if (!(P.layers[st.layer].tags & BM_TAG_SPATIAL)) return false;
    if (st.kind == ST_TUFT) return A->fused.t[st.layer][st.idx].ok;
    return st.kind == ST_INHIB_MTP;
}

// What a frame intake writes: the axon slices of every input.
StepAccess intake_access(const bm_area_plan& P) {
    StepAccess a;
    for (uint32_t i = 0; i < P.n_inputs; i++) {
        const uint64_t b = P.inputs[i].axn_idz, e = b + P.inputs[i].len;
        for (uint32_t s = 0; s < P.n_slices && s < BM_MAX_SLICES; s++) {
            const uint64_t sb = P.slc_axn_idz[s], se = sb + (uint64_t)P.slc_v_size[s] * P.slc_u_size[s];
            if (sb < e && b < se) a.ax_w.set(s);
        }
    }
    return a;
}

void free_front_events(bm_area_s* A) {
    for (cudaEvent_t ev : A->front_ev)
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : A->main_ev)
        if (ev) cudaEventDestroy(ev);
    A->front_ev.clear();
    A->main_ev.clear();
}

// The front stream's part of the schedule (see bm_area_s::front_n): the
// leading steps front_step_ok takes (at least one step must stay behind), the
// previous cycle's steps each waits for (the cycle end excepted: front kernels
// do not read the counter), the front steps each later step waits for, and
// the intake's waits both ways. Filtered inputs keep the program's first step
// a filter, so such areas have no front stream.
int schedule_front(bm_area_s* A, const std::vector<StepAccess>& acc) {
    const size_t n = A->steps.size();
    free_front_events(A);
    A->front_n = 0;
    A->front_prev.clear();
    A->front_waits.clear();
    A->intake_prev.clear();
    A->intake_readers.clear();
    A->main_ev_needed.clear();
    A->front_ax_w.reset();
    size_t f = 0;
    if (A->exec_path == BM_PATH_FUSED)
        while (f < n && front_step_ok(A, A->steps[f])) f++;
    // Work already queued on the main stream comes before the front stream's
    // next steps (the new events have no records yet).
    A->mark_main();
    if (f == 0 || f >= n) return BM_OK;
    A->front_prev.assign(f, {});
    A->front_waits.assign(n, {});
    A->main_ev_needed.assign(n, 0);
    A->intake_readers.assign(n, 0);
    for (size_t k = 0; k < f; k++) A->front_ax_w |= acc[k].ax_w;
    const StepAccess in = intake_access(A->plan);
    for (size_t t = f; t < n; t++) {
        const bool counter_only = A->steps[t].kind == ST_CYCLE_END;
        for (size_t k = 0; k < f; k++) {
            if (!counter_only && conflict(acc[t], acc[k])) {
                A->front_prev[k].push_back(t);
                if (!A->step_side[t]) A->main_ev_needed[t] = 1;
            }
            if (conflict(acc[k], acc[t])) A->front_waits[t].push_back(k);
        }
        if (!counter_only && conflict(in, acc[t])) {
            A->intake_prev.push_back(t);
            if (!A->step_side[t]) A->main_ev_needed[t] = 1;
            A->intake_readers[t] = 1;
        }
    }
    cudaError_t e = cudaSuccess;
    if (!A->front) e = stream_like(A->stream(), &A->front);
    if (e == cudaSuccess && !A->intake_ev) e = cudaEventCreateWithFlags(&A->intake_ev, cudaEventDisableTiming);
    if (e == cudaSuccess && !A->main_mark) e = cudaEventCreateWithFlags(&A->main_mark, cudaEventDisableTiming);
    A->front_ev.assign(f, nullptr);
    A->main_ev.assign(n, nullptr);
    for (size_t k = 0; k < f && e == cudaSuccess; k++) e = cudaEventCreateWithFlags(&A->front_ev[k], cudaEventDisableTiming);
    for (size_t t = 0; t < n && e == cudaSuccess; t++)
        if (A->main_ev_needed[t]) e = cudaEventCreateWithFlags(&A->main_ev[t], cudaEventDisableTiming);
    if (e != cudaSuccess) {
        free_front_events(A);
        return cuda_err(e, "front stream");
    }
    A->front_n = f;
    return BM_OK;
}

}  // namespace

// Front stream in use: scheduled, not profiling, and no sampler reading an
// axon slice the front steps write (or anything but axons): a sampler's copy
// follows its cycle on the main stream, and the next cycle's front steps
// could otherwise overwrite the range before it is taken.
bool bm_area_s::front_active() const {
    if (!front_n || profiling || !front) return false;
    for (const bm_sampler_s* S : samplers) {
        uint64_t off, len;
        sampler_range(S, &off, &len);
        if (off < plan.axon_off || off + len > plan.axon_off + plan.n_axons) return false;
        for (uint32_t s = 0; s < plan.n_slices && s < BM_MAX_SLICES; s++) {
            if (!front_ax_w.test(s)) continue;
            const uint64_t b = plan.axon_off + plan.slc_axn_idz[s];
            const uint64_t e = b + (uint64_t)plan.slc_v_size[s] * plan.slc_u_size[s];
            if (b < off + len && off < e) return false;
        }
    }
    return true;
}

int bm::schedule_area(bm_area_s* A) {
    const size_t n = A->steps.size();
    std::vector<StepAccess> acc(n);
    for (size_t k = 0; k < n; k++) acc[k] = step_access(A, A->steps[k]);
    A->step_side.assign(n, 0);
    A->step_waits.assign(n, {});
    A->last_side = SIZE_MAX;
    for (size_t k = 0; k < n; k++) {
        const uint8_t kind = A->steps[k].kind;
        if (kind != ST_TUFT && kind != ST_TUFTS_PLAIN) continue;
        bool free = true;
        for (size_t j = 0; j < k && free; j++)
            if (!A->step_side[j] && conflict(acc[j], acc[k])) free = false;
        A->step_side[k] = free;
    }
    for (size_t k = 0; k < n; k++) {
        if (A->step_side[k]) {
            A->last_side = k;
            continue;
        }
        for (size_t j = 0; j < k; j++)
            if (A->step_side[j] && conflict(acc[j], acc[k])) A->step_waits[k].push_back(j);
    }
    // The cycle-end launch folds into a final pyramidal tail on the main
    // stream once every side step has joined the main stream by then (so no
    // step of the cycle reads the cycle number after it advances). The side
    // stream runs its steps in order, so a main step's wait for side step j
    // joins every side step up to j.
    A->end_in_tail = false;
    if (n >= 2 && A->steps[n - 1].kind == ST_CYCLE_END && A->steps[n - 2].kind == ST_PYR_TAIL && !A->step_side[n - 2]) {
        size_t joined = 0;   // side steps below this index have joined
        for (size_t k = 0; k + 1 < n; k++)
            if (!A->step_side[k])
                for (size_t j : A->step_waits[k]) joined = std::max(joined, j + 1);
        A->end_in_tail = A->last_side == SIZE_MAX || A->last_side < joined;
    }
    for (cudaEvent_t ev : A->side_ev)
        if (ev) cudaEventDestroy(ev);
    A->side_ev.clear();
    cudaError_t e = cudaSuccess;
    if (A->last_side != SIZE_MAX) {
        if (!A->side) e = stream_like(A->stream(), &A->side);
        if (e == cudaSuccess && !A->ev_fork) e = cudaEventCreateWithFlags(&A->ev_fork, cudaEventDisableTiming);
        A->side_ev.assign(n, nullptr);
        for (size_t k = 0; k < n && e == cudaSuccess; k++)
            if (A->step_side[k]) e = cudaEventCreateWithFlags(&A->side_ev[k], cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_err(e, "side stream");
    }
    return schedule_front(A, acc);
}

void bm::run_pending_verifies(bm_area_s* A, cudaStream_t s) {
    bool any = false;
    for (uint32_t i = 0; i < A->plan.n_layers; i++)
        if (A->verify_pending[i]) {
            launch_verify_tufts(A->fused, A->dl[i], i, A->ctl, s);
            A->verify_pending[i] = false;
            any = true;
        }
    // Regrowth keeps the compiled gather offsets current: it needs each
    // tuft's footprint geometry as last planned (retiling changes it).
    if (any && A->d_geo) {
        refresh_geo(A);
        cudaMemcpyAsync(A->d_geo, A->geo, sizeof A->geo, cudaMemcpyHostToDevice, s);
    }
}

void bm::refresh_geo(bm_area_s* A) {
    for (uint32_t i = 0; i < A->plan.n_layers; i++)
        for (uint32_t t = 0; t < A->plan.layers[i].n_tufts; t++) {
            const FusedTuft& FT = A->fused.t[i][t];
            TuftGeo& G = A->geo[i][t];
            const bool tiled = A->exec_path == BM_PATH_FUSED && FT.ok && FT.tiled && FT.gidx;
            G.gidx = tiled ? FT.gidx : nullptr;
            G.g = gather_geo(A->fused, A->plan, i, t);
            G.tiled = tiled;
        }
}

namespace {

// Makes stream s wait for step t's event of the latest cycle that recorded it
// (a side step's, or a main step's the front stream depends on).
void wait_step(bm_area_s* A, size_t t, cudaStream_t s) {
    if (A->last_side != SIZE_MAX && A->step_side[t]) cudaStreamWaitEvent(s, A->side_ev[t], 0);
    else if (t < A->main_ev.size() && A->main_ev[t]) cudaStreamWaitEvent(s, A->main_ev[t], 0);
}

// Before front-stream work (an intake, or a cycle's front steps): after the
// main stream's marked position, and after everything queued on the main
// stream when the latest cycle did not use the front stream (nothing recorded
// the events the front stream's waits refer to).
void front_begin(bm_area_s* A) {
    if (!A->front_last) A->mark_main();
    cudaStreamWaitEvent(A->front, A->main_mark, 0);
}

// The stream a frame intake goes to, with its waits on the previous cycle
// when that is the front stream.
cudaStream_t intake_begin(bm_area_s* A) {
    if (!A->front_active()) return A->stream();
    front_begin(A);
    for (size_t t : A->intake_prev) wait_step(A, t, A->front);
    return A->front;
}

// After an intake's copies: later steps reading the inputs follow it, and with
// `join` the main stream does too (an intake outside a cycling call).
void intake_end(bm_area_s* A, cudaStream_t s, bool join) {
    if (s != A->front) return;
    cudaEventRecord(A->intake_ev, s);
    if (join) cudaStreamWaitEvent(A->stream(), A->intake_ev, 0);
}

int enqueue_cycle(bm_area_s* A) {
    A->launches = 0;
    cudaStream_t main = A->stream();
    bool verify = false;
    for (uint32_t i = 0; i < A->plan.n_layers; i++) verify = verify || A->verify_pending[i];
    run_pending_verifies(A, main);
    const bool front = A->front_active();
    if (front && verify) A->mark_main();   // the compiled offsets the front steps read
    const size_t nf = front ? A->front_n : 0;
    // Profiling times each launch on its own: everything on the main stream.
    size_t last_side = SIZE_MAX;
    for (size_t k = nf; k < A->steps.size() && !A->profiling; k++)
        if (A->step_side[k]) last_side = k;
    const bool fork = last_side != SIZE_MAX;
    if (front) {
        front_begin(A);
        for (size_t k = 0; k < nf; k++) {
            for (size_t t : A->front_prev[k]) wait_step(A, t, A->front);
            exec_step(A, A->steps[k], A->front, false);
            cudaEventRecord(A->front_ev[k], A->front);
        }
    }
    if (fork) {
        cudaEventRecord(A->ev_fork, main);
        cudaStreamWaitEvent(A->side, A->ev_fork, 0);
    }
    // With end_in_tail the last pyramidal tail ends the cycle itself and the
    // cycle-end step (the last) launches nothing.
    const size_t n = A->steps.size() - (A->end_in_tail ? 1 : 0);
    const bool regrow_fires = A->host_cycle % kRegrowPeriod == kRegrowPeriod - 1;
    for (size_t k = nf; k < n; k++) {
        const bool on_side = fork && A->step_side[k];
        cudaStream_t s = on_side ? A->side : main;
        if (fork && !on_side)
            for (size_t j : A->step_waits[k])
                if (j >= nf) cudaStreamWaitEvent(main, A->side_ev[j], 0);
        if (front) {
            for (size_t j : A->front_waits[k]) cudaStreamWaitEvent(s, A->front_ev[j], 0);
            if (A->intake_readers[k]) cudaStreamWaitEvent(s, A->intake_ev, 0);
        }
        exec_step(A, A->steps[k], s, A->end_in_tail && k + 1 == n);
        if (on_side) cudaEventRecord(A->side_ev[k], A->side);
        else if (front && A->main_ev_needed[k] && (A->steps[k].kind != ST_REGROW || regrow_fires))
            cudaEventRecord(A->main_ev[k], main);
    }
    if (fork) cudaStreamWaitEvent(main, A->side_ev[last_side], 0);
    if (front) cudaStreamWaitEvent(main, A->front_ev[nf - 1], 0);
    A->front_last = front;
    A->host_cycle++;
    return A->samplers.empty() ? BM_OK : sample_after_cycle(A, main);
}

bool buf_range(bm_area_s* A, uint32_t kind, uint32_t layer, uint64_t offset, uint64_t len, uint64_t* off_out) {
    const bm_area_plan& P = A->plan;
    if (kind == BM_BUF_AXON_STATES) {
        if (offset > P.n_axons || len > P.n_axons - offset) return false;
        *off_out = P.axon_off + offset;
        return true;
    }
    if (kind >= BM_BUF_COUNT || layer >= P.n_layers) return false;
    const bm_layer_plan& L = P.layers[layer];
    if (L.buf_off[kind] == UINT64_MAX) return false;
    if (offset > L.buf_len[kind] || len > L.buf_len[kind] - offset) return false;
    *off_out = L.buf_off[kind] + offset;
    return true;
}

}  // namespace

void bm::fill_dev_layer(DevLayer& D, const bm_area_plan& P, uint32_t i, uint8_t* slab) {
    const bm_layer_plan& L = P.layers[i];
    std::memset(&D, 0, sizeof D);
    D.kind = L.kind;
    D.depth = L.depth;
    D.v_size = L.v_size;
    D.u_size = L.u_size;
    D.cells = L.cells;
    D.base_slc = L.base_axn_slc;
    D.axn_idz = L.axn_idz;
    D.n_tufts = L.n_tufts;
    D.enabled_flags = L.enabled_tft_flags;
    D.prx_id = L.bsl_prx_tft_id;
    D.dst_id = L.bsl_dst_tft_id;
    D.apc_id = L.apc_dst_tft_id;
    D.n_syns = L.n_syns;
    for (int k = 0; k < BM_BUF_COUNT; k++)
        D.buf[k] = L.buf_off[k] == UINT64_MAX ? nullptr : slab + L.buf_off[k];
    for (uint32_t t = 0; t < L.n_tufts; t++) {
        const bm_tuft_plan& T = L.tufts[t];
        DevTuft& DT = D.tft[t];
        DT.dpt = T.dens_per_tft;
        DT.spd = T.syns_per_den;
        DT.spt = T.syns_per_tft;
        DT.mad_l2 = T.max_active_dens_l2;
        DT.thresh = T.den_threshold;
        DT.den_kind = T.den_kind;
        DT.syn_idz = T.syn_idz;
        DT.den_idz = T.den_idz;
        DT.cel_idz = T.cel_idz;
        DT.rnd_key_den = rnd_key(P.rnd_seed, P.area_id, L.layer_id, BM_RND_DEN_CYCLE, t);
        DT.rnd_key_mtp = rnd_key(P.rnd_seed, P.area_id, L.layer_id, BM_RND_TFT_DST_MTP, t);
    }
    D.rnd_key_ssc_mtp = rnd_key(P.rnd_seed, P.area_id, L.layer_id, BM_RND_SSC_MTP, 0);
}

void bm::fill_slice_table(const bm_area_plan& P, SliceRec* out) {
    for (uint32_t k = 0; k < BM_MAX_SLICES; k++) {
        SliceRec r{0, 0, 0, 0};
        if (k < P.n_slices) {
            r.x = P.slc_axn_idz[k];
            r.y = P.slc_v_size[k] | (P.slc_u_size[k] << 16);
            r.z = P.slc_v_scale[k] | (P.slc_u_scale[k] << 8) | (P.slc_v_mid[k] << 16) | (P.slc_u_mid[k] << 24);
        }
        out[k] = r;
    }
}

namespace {

void build_dev_layers(bm_area_s* A) {
    const bm_area_plan& P = A->plan;
    for (uint32_t i = 0; i < P.n_layers; i++) {
        const bm_layer_plan& L = P.layers[i];
        fill_dev_layer(A->dl[i], P, i, A->slab);
        for (uint32_t k = 0; k < L.n_ctrl; k++)
            A->inhib_key[i][k] = rnd_key(P.rnd_seed, P.area_id, L.ctrl[k].layer_id, BM_RND_INHIB, 0);
    }
}

// Regrowth jobs of A: every tuft of every data layer, layers in cycle order
// (CorticalArea::regrow, src/cortex/cortical_area.rs:792-806), each tuft's
// stream keyed by its growth key.
int prepare_regrow(bm_area_s* A, const std::vector<TuftGrowSpec>& grow, const std::vector<GrowTuft>& gts) {
    const bm_area_plan& P = A->plan;
    cudaError_t e = dev_alloc(A->ctx, &A->d_geo, sizeof A->geo);
    if (e != cudaSuccess) return cuda_err(e, "regrowth geometry");
    refresh_geo(A);
    e = cudaMemcpyAsync(A->d_geo, A->geo, sizeof A->geo, cudaMemcpyHostToDevice, A->stream());
    if (e != cudaSuccess) return cuda_err(e, "regrowth geometry");
    uint64_t blocks = 0;
    for (uint32_t k = 0; k < P.n_cycle_order; k++) {
        const uint32_t i = P.cycle_order[k];
        for (size_t g = 0; g < grow.size(); g++) {
            if (grow[g].data_layer != i) continue;
            const uint32_t t = grow[g].tft;
            const uint64_t n = (uint64_t)P.layers[i].cells * P.layers[i].tufts[t].dens_per_tft;
            if (!n) continue;
            if (n > 0xFFFFFFFFull) return set_err(BM_ERR_UNSUPPORTED, "regrowth of more than 2^32 dendrites in a tuft");
            RegrowJob J;
            std::memset(&J, 0, sizeof J);
            J.L = A->dl[i];
            J.G = gts[g];
            J.ctl = A->ctl;
            J.geo = A->d_geo + i * BM_MAX_TUFTS + t;
            J.rkey = regrow_key(grow[g].key);
            J.saturated = grow[g].saturated;
            J.n = (uint32_t)n;
            J.block0 = (uint32_t)blocks;
            blocks += (n + kRegrowBlock - 1) / kRegrowBlock;
            A->regrow.push_back(J);
        }
    }
    if (blocks > 0x7FFFFFFFull) return set_err(BM_ERR_UNSUPPORTED, "regrowth launch of too many blocks");
    if (A->regrow.empty()) return BM_OK;
    e = dev_alloc(A->ctx, &A->d_regrow, A->regrow.size() * sizeof(RegrowJob));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(A->d_regrow, A->regrow.data(), A->regrow.size() * sizeof(RegrowJob),
                            cudaMemcpyHostToDevice, A->stream());
    if (e != cudaSuccess) return cuda_err(e, "regrowth jobs");
    A->regrow_blocks = (uint32_t)blocks;
    return BM_OK;
}

// The host-frame upload ring (bm_area_s::up*).
void free_upload(bm_area_s* A) {
    for (int k = 0; k < 2; k++) {
        if (A->up_host[k]) cudaFreeHost(A->up_host[k]);
        if (A->up_dev[k]) cudaFree(A->up_dev[k]);
        if (A->up_loaded[k]) cudaEventDestroy(A->up_loaded[k]);
        if (A->up_taken[k]) cudaEventDestroy(A->up_taken[k]);
        A->up_host[k] = A->up_dev[k] = nullptr;
        A->up_loaded[k] = A->up_taken[k] = nullptr;
    }
    if (A->up) cudaStreamDestroy(A->up);
    A->up = nullptr;
    A->up_cap = 0;
}

}  // namespace

namespace {
// Page-locked, device-mapped words handed out one at a time (bm::host_word_get).
struct HostWords {
    std::mutex mu;
    std::vector<unsigned int*> free;
};
HostWords& host_words() {
    static HostWords* w = new HostWords;   // kept for the process
    return *w;
}
constexpr size_t kHostWordBlock = 1024;
}  // namespace

cudaError_t bm::host_word_get(unsigned int** host, unsigned int** dev) {
    HostWords& W = host_words();
    std::lock_guard<std::mutex> lk(W.mu);
    if (W.free.empty()) {
        unsigned int* blk = nullptr;
        const cudaError_t e = cudaHostAlloc((void**)&blk, kHostWordBlock * sizeof(unsigned int),
                                            cudaHostAllocMapped | cudaHostAllocPortable);
        if (e != cudaSuccess) return e;
        for (size_t k = kHostWordBlock; k-- > 0;) W.free.push_back(blk + k);
    }
    unsigned int* h = W.free.back();
    const cudaError_t e = cudaHostGetDevicePointer((void**)dev, h, 0);
    if (e != cudaSuccess) return e;
    W.free.pop_back();
    *(volatile unsigned int*)h = 0;
    *host = h;
    return cudaSuccess;
}

void bm::host_word_put(unsigned int* host) {
    HostWords& W = host_words();
    std::lock_guard<std::mutex> lk(W.mu);
    W.free.push_back(host);
}

void bm::ctx_release(bm_ctx c) {
    if (!c || c->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
    DevGuard g(c->device);
    if (c->own) { cudaStreamSynchronize(c->own); cudaStreamDestroy(c->own); }
    delete c;
}

namespace {

void free_area(bm_area_s* A) {
    if (!A) return;
    if (A->ctx) {
        DevGuard g(A->ctx->device);
        // Batches and samplers first: they may still use the memory on their
        // own streams. Pooled memory is then freed in order on the area's
        // stream, which every cycle of the area ends on.
        detach_from_batches(A);
        free_samplers(A);
        free_upload(A);
        const bool pl = A->pooled;
        cudaStream_t s = A->stream();
        dev_free(A->slab, pl, s);
        dev_free(A->ctl, pl, s);
        if (A->host_err) host_word_put(A->host_err);
        dev_free(A->slices, pl, s);
        if (A->down) cudaStreamDestroy(A->down);
        free_fused(A->fused, s);
        dev_free(A->d_regrow, pl, s);
        dev_free(A->grow_offs, pl, s);
        dev_free(A->d_geo, pl, s);
        for (auto& row : A->d_centers)
            for (int32_t* c : row) dev_free(c, pl, s);
        if (A->side) cudaStreamDestroy(A->side);
        if (A->ev_fork) cudaEventDestroy(A->ev_fork);
        free_front_events(A);
        if (A->front) cudaStreamDestroy(A->front);
        if (A->intake_ev) cudaEventDestroy(A->intake_ev);
        if (A->main_mark) cudaEventDestroy(A->main_mark);
        for (cudaEvent_t e : A->side_ev)
            if (e) cudaEventDestroy(e);
        for (auto& r : A->pending) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
        for (auto e : A->pool) cudaEventDestroy(e);
    }
    ctx_release(A->ctx);
    delete A;
}

}  // namespace

void bm::frame_pieces(bm_area_s* A, uint32_t input, uint32_t off, uint32_t len, std::vector<FramePiece>& out) {
    const bm_area_plan& P = A->plan;
    out.clear();
    uint8_t* axons = A->axns() + P.inputs[input].axn_idz;
    const bool filtered = filters_run(P);
    const uint32_t end = off + len;
    uint32_t pos = off;
    while (pos < end) {
        const bm_filter_chain_plan* hit = nullptr;
        uint32_t next = end;
        for (uint32_t k = 0; filtered && k < P.n_filter_chains; k++) {
            const bm_filter_chain_plan& c = P.filter_chains[k];
            if (c.input != input) continue;
            const uint32_t c0 = c.frame_off, c1 = c0 + c.depth * c.v_size * c.u_size;
            if (pos >= c0 && pos < c1) {
                hit = &c;
                next = std::min(end, c1);
            } else if (!hit && c0 > pos && c0 < next) {
                next = c0;
            }
        }
        out.push_back({pos - off, next - pos, hit ? A->slab + hit->buf_off[0] + (pos - hit->frame_off) : axons + pos});
        pos = next;
    }
}

namespace {

// Copies one input frame to where its pieces land (see frame_pieces).
// Copies of frame pieces on stream s: device-to-device ones as one copy
// kernel launched like the cycle's kernels (see CopyPieces).
int copy_pieces(const std::vector<FramePiece>& pieces, const uint8_t* src, cudaMemcpyKind kind, cudaStream_t s) {
    if (kind == cudaMemcpyDeviceToDevice && !pieces.empty() && pieces.size() <= kMaxCopyPieces) {
        CopyPieces P = {};
        for (const FramePiece& p : pieces) {
            P.dst[P.n] = p.dst;
            P.src[P.n] = src + p.off;
            P.len[P.n] = p.len;
            P.n++;
        }
        launch_copy_pieces(P, s);
        CU(cudaGetLastError());
        return BM_OK;
    }
    for (const FramePiece& p : pieces) CU(cudaMemcpyAsync(p.dst, src + p.off, p.len, kind, s));
    return BM_OK;
}

int write_frame(bm_area_s* A, uint32_t input, const void* src, cudaMemcpyKind kind, cudaStream_t s) {
    std::vector<FramePiece> pieces;
    frame_pieces(A, input, 0, A->plan.inputs[input].len, pieces);
    return copy_pieces(pieces, (const uint8_t*)src, kind, s);
}

// A host frame: the caller's bytes are read during the call only, into a
// pinned slot; the slot is uploaded on A->up (beside the cycles still
// running on the area's stream) and then moved into place on the area's
// stream, ordered before the next cycle as a direct copy would be.
int write_host_frame(bm_area_s* A, uint32_t input, const uint8_t* frame, size_t len) {
    cudaError_t e = cudaSuccess;
    if (!A->up) {
        size_t cap = 0;
        for (uint32_t i = 0; i < A->plan.n_inputs; i++) cap = std::max<size_t>(cap, A->plan.inputs[i].len);
        for (int k = 0; k < 2 && e == cudaSuccess; k++) {
            e = cudaHostAlloc((void**)&A->up_host[k], cap, cudaHostAllocDefault);
            if (e == cudaSuccess) e = cudaMalloc(&A->up_dev[k], cap);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&A->up_loaded[k], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&A->up_taken[k], cudaEventDisableTiming);
        }
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&A->up, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            free_upload(A);
            return cuda_err(e, "input upload set-up");
        }
        A->up_cap = cap;
        A->up_next = 0;
    }
    if (len > A->up_cap) return set_err(BM_ERR_INVALID, "frame of %zu bytes exceeds the upload slot", len);
    const uint32_t k = A->up_next;
    A->up_next ^= 1;
    // The slot's previous upload has finished reading its pinned bytes.
    e = cudaEventSynchronize(A->up_loaded[k]);
    if (e != cudaSuccess) return cuda_err(e, "input upload");
    std::memcpy(A->up_host[k], frame, len);
    // The area's stream has moved the slot's previous frame into place.
    e = cudaStreamWaitEvent(A->up, A->up_taken[k], 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(A->up_dev[k], A->up_host[k], len, cudaMemcpyHostToDevice, A->up);
    if (e == cudaSuccess) e = cudaEventRecord(A->up_loaded[k], A->up);
    const cudaStream_t s = intake_begin(A);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, A->up_loaded[k], 0);
    if (e != cudaSuccess) return cuda_err(e, "input upload");
    const int rc = write_frame(A, input, A->up_dev[k], cudaMemcpyDeviceToDevice, s);
    if (rc != BM_OK) return rc;
    e = cudaEventRecord(A->up_taken[k], s);
    intake_end(A, s, true);
    return e == cudaSuccess ? BM_OK : cuda_err(e, "input upload");
}

}  // namespace

extern "C" {

const char* bm_last_error(void) { return g_err; }

const char* bm_version(void) { return "bismit_b200 0.1 (sm_100a)"; }

int32_t bm_rnd(uint64_t seed, uint32_t area_id, uint32_t layer_id, uint32_t role, uint32_t tft_id, uint64_t cycle) {
    return rnd_at(rnd_key(seed, area_id, layer_id, role, tft_id), cycle);
}

int bm_ctx_create(int device, uint32_t flags, bm_ctx* out) {
    (void)flags;
    if (!out) return set_err(BM_ERR_INVALID, "bm_ctx_create: null out");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return set_err(BM_ERR_NO_DEVICE, "no CUDA device (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= n) return set_err(BM_ERR_NO_DEVICE, "device %d out of range (%d devices)", device, n);
    DevGuard g(device);
    bm_ctx c = new (std::nothrow) bm_ctx_s;
    if (!c) return set_err(BM_ERR_OOM, "host allocation failed");
    c->device = device;
    e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete c; return cuda_err(e, "cudaStreamCreate"); }
    *out = c;
    return BM_OK;
}

int bm_ctx_destroy(bm_ctx ctx) {
    if (!ctx) return BM_OK;
    ctx_release(ctx);
    return BM_OK;
}

int bm_ctx_set_stream(bm_ctx ctx, void* stream) {
    if (!ctx) return set_err(BM_ERR_INVALID, "null ctx");
    ctx->user = (cudaStream_t)stream;
    ctx->user_set = true;
    return BM_OK;
}

int bm_ctx_use_own_stream(bm_ctx ctx) {
    if (!ctx) return set_err(BM_ERR_INVALID, "null ctx");
    ctx->user = nullptr;
    ctx->user_set = false;
    return BM_OK;
}

int bm_ctx_synchronize(bm_ctx ctx) {
    if (!ctx) return set_err(BM_ERR_INVALID, "null ctx");
    DevGuard g(ctx->device);
    CU(cudaStreamSynchronize(ctx->stream()));
    return BM_OK;
}

int bm_area_create(bm_ctx ctx, const bm_area_desc* desc, uint64_t seed, bm_area* out) {
    if (!ctx || !desc || !out) return set_err(BM_ERR_INVALID, "bm_area_create: null argument");
    *out = nullptr;
    DevGuard g(ctx->device);
    bm_area_s* A = new (std::nothrow) bm_area_s;
    if (!A) return set_err(BM_ERR_OOM, "host allocation failed");
    std::vector<TuftGrowSpec> grow;
    std::string err;
    int rc = resolve_area(desc, seed, &A->plan, &grow, &err);
    if (rc != BM_OK) { delete A; return set_err(rc, "%s", err.c_str()); }
    A->exec_path = desc->exec_path;
    if (A->exec_path != BM_PATH_FUSED && A->exec_path != BM_PATH_PLAIN) {
        delete A;
        return set_err(BM_ERR_INVALID, "unknown exec_path %u", desc->exec_path);
    }
    A->ctx = ctx;
    ctx_retain(ctx);
    A->pooled = ctx->pool != nullptr;
    A->fused.pool = ctx->pool;
    A->fused.pool_stream = ctx->stream();
    cudaStream_t s = ctx->stream();
    cudaError_t e = dev_alloc(ctx, &A->slab, A->plan.slab_bytes);
    if (e != cudaSuccess) {
        free_area(A);
        return set_err(BM_ERR_OOM, "cudaMalloc of %llu state bytes failed: %s",
                       (unsigned long long)A->plan.slab_bytes, cudaGetErrorString(e));
    }
    e = dev_alloc(ctx, &A->ctl, sizeof(AreaCtl));
    if (e == cudaSuccess) e = dev_alloc(ctx, &A->slices, sizeof(SliceRec) * BM_MAX_SLICES);
    if (e != cudaSuccess) { free_area(A); return cuda_err(e, "cudaMalloc"); }
    std::vector<SliceRec> tab(BM_MAX_SLICES);
    fill_slice_table(A->plan, tab.data());
    AreaCtl ctl0{};
    unsigned int* dev_err = nullptr;
    e = host_word_get(&A->host_err, &dev_err);
    if (e != cudaSuccess) { free_area(A); return cuda_err(e, "host-mapped error word"); }
    ctl0.host_err = dev_err;
    e = cudaMemsetAsync(A->slab, 0, A->plan.slab_bytes, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(A->slices, tab.data(), sizeof(SliceRec) * BM_MAX_SLICES, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(A->ctl, &ctl0, sizeof ctl0, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) { free_area(A); return cuda_err(e, "area init copy"); }
    build_dev_layers(A);

    // Growth (Synapses::grow(true)): offset pools to the device, one launch per tuft.
    std::vector<int8_t> ov, ou;
    for (auto& G : grow)
        for (auto& S : G.srcs) { ov.insert(ov.end(), S.offs_v.begin(), S.offs_v.end()); ou.insert(ou.end(), S.offs_u.begin(), S.offs_u.end()); }
    int8_t* d_off = nullptr;
    size_t n_off = ov.size();
    if (n_off) {
        e = dev_alloc(ctx, &d_off, 2 * n_off);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_off, ov.data(), n_off, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_off + n_off, ou.data(), n_off, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) { dev_free(d_off, A->pooled, s); free_area(A); return cuda_err(e, "growth pools"); }
    }
    uint32_t base = 0;
    std::vector<GrowTuft> gts;
    for (auto& G : grow) {
        GrowTuft GT;
        std::memset(&GT, 0, sizeof GT);
        GT.tft = G.tft;
        GT.key = G.key;
        GT.n_pool = G.n_pool;
        std::memcpy(GT.pool, G.pool, sizeof GT.pool);
        std::memcpy(GT.pool_src, G.pool_src, sizeof GT.pool_src);
        for (size_t k = 0; k < G.srcs.size(); k++) {
            GT.nonspatial[k] = G.srcs[k].nonspatial;
            GT.rv[k] = G.srcs[k].rv;
            GT.ru[k] = G.srcs[k].ru;
            GT.n_offs[k] = (uint32_t)G.srcs[k].offs_v.size();
            GT.offs_base[k] = base;
            base += GT.n_offs[k];
        }
        GT.offs_v = d_off;
        GT.offs_u = d_off ? d_off + n_off : nullptr;
        GT.unique = !(desc->init_flags & BM_INIT_NO_UNIQUE) && !G.saturated;
        GT.zero_strength = (desc->init_flags & BM_INIT_STRENGTH_ZERO) != 0;
        launch_grow(A->dl[G.data_layer], GT, s);
        gts.push_back(GT);
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    const bool regrow = !(A->plan.settings & BM_SET_DISABLE_REGROWTH);
    if (regrow) A->grow_offs = d_off;   // kept: regrowth draws from the same pools
    else dev_free(d_off, A->pooled, s);
    if (e != cudaSuccess) { free_area(A); return cuda_err(e, "synapse growth"); }
    rc = prepare_fused(A->fused, A->plan, &err);
    if (rc == BM_OK) rc = bind_fused(A->fused, A->plan, A->axns());
    if (rc != BM_OK) { free_area(A); return set_err(rc, "%s", err.c_str()); }
    if (regrow) {
        rc = prepare_regrow(A, grow, gts);
        if (rc != BM_OK) { free_area(A); return rc; }
    }
    // Activity smoothers' group centers.
    for (uint32_t i = 0; i < A->plan.n_layers; i++) {
        const bm_layer_plan& L = A->plan.layers[i];
        for (uint32_t k = 0; k < L.n_ctrl; k++) {
            if (L.ctrl[k].kind != BM_LYR_CTRL_SMOOTHER) continue;
            std::vector<int32_t> c;
            smoother_centers((int)L.ctrl[k].field_radius, (int)L.v_size, (int)L.u_size, c, A->center_off[i][k]);
            e = dev_alloc(ctx, &A->d_centers[i][k], std::max<size_t>(1, c.size()) * sizeof(int32_t));
            if (e == cudaSuccess && !c.empty())
                e = cudaMemcpyAsync(A->d_centers[i][k], c.data(), c.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                    s);
            if (e != cudaSuccess) { free_area(A); return cuda_err(e, "smoother centers"); }
        }
    }
    for (uint32_t i = 0; i < A->plan.n_layers; i++) A->verify_pending[i] = true;
    area_steps(A, A->steps, cell_tuft_cells(A) <= kFoldCellTufts);
    rc = schedule_area(A);
    if (rc != BM_OK) { free_area(A); return rc; }
    // Tables copied up in order on the creating stream are in place before
    // the area is cycled on whatever stream the context has then.
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { free_area(A); return cuda_err(e, "area set-up"); }
    *out = A;
    return BM_OK;
}

int bm_area_destroy(bm_area area) {
    if (!area) return BM_OK;
    {
        DevGuard g(area->ctx->device);
        cudaStreamSynchronize(area->stream());
    }
    free_area(area);
    return BM_OK;
}

int bm_area_get_plan(bm_area area, bm_area_plan* out) {
    if (!area || !out) return set_err(BM_ERR_INVALID, "null argument");
    *out = area->plan;
    return BM_OK;
}

int bm_plan_resolve(const bm_area_desc* desc, uint64_t seed, bm_area_plan* out) {
    if (!desc || !out) return set_err(BM_ERR_INVALID, "null argument");
    std::string err;
    int rc = resolve_area(desc, seed, out, nullptr, &err);
    if (rc != BM_OK) return set_err(rc, "%s", err.c_str());
    return BM_OK;
}

int bm_area_write_input(bm_area area, uint32_t input_idx, const uint8_t* frame, size_t len) {
    if (!area || !frame) return set_err(BM_ERR_INVALID, "null argument");
    const bm_area_plan& P = area->plan;
    if (input_idx >= P.n_inputs) return set_err(BM_ERR_INVALID, "input %u out of range (%u inputs)", input_idx, P.n_inputs);
    if (len != P.inputs[input_idx].len)
        return set_err(BM_ERR_INVALID, "frame length %zu != input layer axon count %u", len, P.inputs[input_idx].len);
    DevGuard g(area->ctx->device);
    return write_host_frame(area, input_idx, frame, len);
}

int bm_area_write_input_device(bm_area area, uint32_t input_idx, const void* dev_frame, size_t len) {
    if (!area || !dev_frame) return set_err(BM_ERR_INVALID, "null argument");
    const bm_area_plan& P = area->plan;
    if (input_idx >= P.n_inputs) return set_err(BM_ERR_INVALID, "input %u out of range", input_idx);
    if (len != P.inputs[input_idx].len) return set_err(BM_ERR_INVALID, "frame length %zu != %u", len, P.inputs[input_idx].len);
    DevGuard g(area->ctx->device);
    const cudaStream_t s = intake_begin(area);
    const int rc = write_frame(area, input_idx, dev_frame, cudaMemcpyDeviceToDevice, s);
    intake_end(area, s, true);
    return rc;
}

namespace {
// A cycle that completed with device error bits stops further cycles of the
// area until bm_area_clear_errors (its state is no longer a cycle's result).
int refuse_after_errors(const bm_area_s* A) {
    const unsigned int e = A->seen_errors();
    if (!e) return BM_OK;
    return set_err(BM_ERR_TIMEOUT,
                   "an earlier cycle of this area ended with device error bits 0x%x (bit 0: a bounded wait gave "
                   "up); bm_area_clear_errors re-enables cycling",
                   e);
}
}  // namespace

int bm_area_cycle(bm_area area, uint32_t n_cycles) {
    if (!area) return set_err(BM_ERR_INVALID, "null area");
    if (int rc = refuse_after_errors(area)) return rc;
    DevGuard g(area->ctx->device);
    for (uint32_t k = 0; k < n_cycles; k++) {
        const int rc = enqueue_cycle(area);
        if (rc != BM_OK) return rc;
    }
    CU(cudaGetLastError());
    return BM_OK;
}

int bm_area_cycle_frames_device(bm_area area, const void* dev_frames, size_t frame_len, uint32_t n_cycles) {
    if (!area || !dev_frames) return set_err(BM_ERR_INVALID, "null argument");
    const bm_area_plan& P = area->plan;
    if (P.n_inputs == 0) return set_err(BM_ERR_INVALID, "area has no input layer");
    if (frame_len != P.inputs[0].len) return set_err(BM_ERR_INVALID, "frame length %zu != %u", frame_len, P.inputs[0].len);
    if (int rc = refuse_after_errors(area)) return rc;
    DevGuard g(area->ctx->device);
    for (uint32_t k = 0; k < n_cycles; k++) {
        int rc = BM_OK;
        area->run(K_INTAKE, [&] {
            const cudaStream_t s = intake_begin(area);
            rc = write_frame(area, 0, (const uint8_t*)dev_frames + (uint64_t)k * frame_len, cudaMemcpyDeviceToDevice,
                             s);
            intake_end(area, s, false);
        });
        if (rc == BM_OK) rc = enqueue_cycle(area);
        if (rc != BM_OK) return rc;
    }
    CU(cudaGetLastError());
    return BM_OK;
}

int bm_area_read_output(bm_area area, uint32_t output_idx, uint8_t* dst, size_t len) {
    if (!area || !dst) return set_err(BM_ERR_INVALID, "null argument");
    const bm_area_plan& P = area->plan;
    if (output_idx >= P.n_outputs) return set_err(BM_ERR_INVALID, "output %u out of range", output_idx);
    if (len != P.outputs[output_idx].len) return set_err(BM_ERR_INVALID, "length %zu != %u", len, P.outputs[output_idx].len);
    DevGuard g(area->ctx->device);
    CU(cudaMemcpyAsync(dst, area->axns() + P.outputs[output_idx].axn_idz, len, cudaMemcpyDeviceToHost, area->stream()));
    CU(cudaStreamSynchronize(area->stream()));
    return BM_OK;
}

int bm_area_read(bm_area area, uint32_t buf_kind, uint32_t layer, uint64_t offset, void* dst, uint64_t len) {
    if (!area || (!dst && len)) return set_err(BM_ERR_INVALID, "null argument");
    uint64_t off;
    if (!buf_range(area, buf_kind, layer, offset, len, &off))
        return set_err(BM_ERR_INVALID, "buffer %u of layer %u: range [%llu, +%llu) out of bounds", buf_kind, layer,
                       (unsigned long long)offset, (unsigned long long)len);
    DevGuard g(area->ctx->device);
    if (len) CU(cudaMemcpyAsync(dst, area->slab + off, len, cudaMemcpyDeviceToHost, area->stream()));
    CU(cudaStreamSynchronize(area->stream()));
    return BM_OK;
}

int bm_area_write(bm_area area, uint32_t buf_kind, uint32_t layer, uint64_t offset, const void* src, uint64_t len) {
    if (!area || (!src && len)) return set_err(BM_ERR_INVALID, "null argument");
    uint64_t off;
    if (!buf_range(area, buf_kind, layer, offset, len, &off))
        return set_err(BM_ERR_INVALID, "buffer %u of layer %u: range out of bounds", buf_kind, layer);
    DevGuard g(area->ctx->device);
    if (len) CU(cudaMemcpyAsync(area->slab + off, src, len, cudaMemcpyHostToDevice, area->stream()));
    CU(cudaStreamSynchronize(area->stream()));
    if (buf_kind == BM_BUF_SYN_SRC_SLC_IDS && len)
        note_sources(area, layer, offset, offset + len, (const uint8_t*)src, false);
    if (buf_kind == BM_BUF_SYN_SRC_SLC_IDS || buf_kind == BM_BUF_SYN_SRC_COL_V_OFFS ||
        buf_kind == BM_BUF_SYN_SRC_COL_U_OFFS || buf_kind == BM_BUF_SYN_FLAG_SETS)
        area->verify_pending[layer] = true;
    return BM_OK;
}

int bm_area_read_slab(bm_area area, void* dst, uint64_t len) {
    if (!area || !dst) return set_err(BM_ERR_INVALID, "null argument");
    if (len != area->plan.slab_bytes) return set_err(BM_ERR_INVALID, "slab length %llu != %llu", (unsigned long long)len,
                                                     (unsigned long long)area->plan.slab_bytes);
    DevGuard g(area->ctx->device);
    CU(cudaMemcpyAsync(dst, area->slab, len, cudaMemcpyDeviceToHost, area->stream()));
    CU(cudaStreamSynchronize(area->stream()));
    return BM_OK;
}

int bm_area_write_slab(bm_area area, const void* src, uint64_t len) {
    if (!area || !src) return set_err(BM_ERR_INVALID, "null argument");
    if (len != area->plan.slab_bytes) return set_err(BM_ERR_INVALID, "slab length mismatch");
    DevGuard g(area->ctx->device);
    CU(cudaMemcpyAsync(area->slab, src, len, cudaMemcpyHostToDevice, area->stream()));
    CU(cudaStreamSynchronize(area->stream()));
    for (uint32_t i = 0; i < area->plan.n_layers; i++) {
        area->verify_pending[i] = true;
        const bm_layer_plan& L = area->plan.layers[i];
        note_sources(area, i, 0, L.n_syns, (const uint8_t*)src + L.buf_off[BM_BUF_SYN_SRC_SLC_IDS], true);
    }
    return BM_OK;
}

int bm_area_sources_changed(bm_area area, uint32_t layer) {
    if (!area || layer >= area->plan.n_layers) return set_err(BM_ERR_INVALID, "bad area or layer");
    area->verify_pending[layer] = true;
    note_sources(area, layer, 0, area->plan.layers[layer].n_syns, nullptr, false);   // written on the device: unknown
    return BM_OK;
}

int bm_area_device_errors(bm_area area, uint32_t* bits) {
    if (!area || !bits) return set_err(BM_ERR_INVALID, "null argument");
    DevGuard g(area->ctx->device);
    unsigned int e = 0;
    CU(cudaMemcpyAsync(&e, &area->ctl->error, sizeof e, cudaMemcpyDeviceToHost, area->stream()));
    CU(cudaStreamSynchronize(area->stream()));
    *bits = e;
    if (e) return set_err(BM_ERR_TIMEOUT, "device-side wait timed out (error bits 0x%x)", e);
    return BM_OK;
}

int bm_area_deliver_tract(bm_area src, uint32_t src_output, bm_area dst, uint32_t dst_input, uint64_t dst_offset) {
    if (!src || !dst) return set_err(BM_ERR_INVALID, "null area");
    if (src->ctx->device != dst->ctx->device) return set_err(BM_ERR_INVALID, "tract between areas on different devices");
    if (src_output >= src->plan.n_outputs) return set_err(BM_ERR_INVALID, "output %u out of range", src_output);
    if (dst_input >= dst->plan.n_inputs) return set_err(BM_ERR_INVALID, "input %u out of range", dst_input);
    const uint32_t len = src->plan.outputs[src_output].len;
    if (dst_offset + len > dst->plan.inputs[dst_input].len)
        return set_err(BM_ERR_INVALID, "tract of %u axons at offset %llu overruns input %u (%u axons)", len,
                       (unsigned long long)dst_offset, dst_input, dst->plan.inputs[dst_input].len);
    DevGuard g(dst->ctx->device);
    cudaStream_t s = dst->stream();
    if (src->stream() != s) {
        // After the work already queued for the source area.
        cudaEvent_t e = src->ev();
        CU(cudaEventRecord(e, src->stream()));
        CU(cudaStreamWaitEvent(s, e, 0));
        src->pool.push_back(e);
    }
    const uint8_t* from = src->axns() + src->plan.outputs[src_output].axn_idz;
    std::vector<FramePiece> pieces;
    frame_pieces(dst, dst_input, (uint32_t)dst_offset, len, pieces);
    const int rc = copy_pieces(pieces, from, cudaMemcpyDeviceToDevice, s);
    dst->mark_main();   // the destination's front steps read its inputs
    if (src->stream() != s) {
        // The source's next cycle overwrites the axons the copy reads.
        cudaEvent_t e = dst->ev();
        CU(cudaEventRecord(e, s));
        CU(cudaStreamWaitEvent(src->stream(), e, 0));
        dst->pool.push_back(e);
    }
    src->mark_main();
    return rc;
}

int bm_area_axons_touched(bm_area area) {
    if (!area) return set_err(BM_ERR_INVALID, "null area");
    DevGuard g(area->ctx->device);
    area->mark_main();
    return BM_OK;
}

int bm_area_clear_errors(bm_area area) {
    if (!area) return set_err(BM_ERR_INVALID, "null area");
    DevGuard g(area->ctx->device);
    const unsigned int zero = 0;
    CU(cudaStreamSynchronize(area->stream()));
    CU(cudaMemcpyAsync(&area->ctl->error, &zero, sizeof zero, cudaMemcpyHostToDevice, area->stream()));
    CU(cudaStreamSynchronize(area->stream()));
    *(volatile unsigned int*)area->host_err = 0;
    return BM_OK;
}

int bm_area_set_wait_limit(bm_area area, uint32_t us) {
    if (!area) return set_err(BM_ERR_INVALID, "null area");
    DevGuard g(area->ctx->device);
    CU(cudaMemcpyAsync(&area->ctl->wait_us, &us, sizeof us, cudaMemcpyHostToDevice, area->stream()));
    CU(cudaStreamSynchronize(area->stream()));
    return BM_OK;
}

int bm_area_inject_stall(bm_area area, uint32_t stage) {
    if (!area) return set_err(BM_ERR_INVALID, "null area");
    DevGuard g(area->ctx->device);
    CU(cudaMemcpyAsync(&area->ctl->stall_stage, &stage, sizeof stage, cudaMemcpyHostToDevice, area->stream()));
    CU(cudaStreamSynchronize(area->stream()));
    return BM_OK;
}

int bm_area_tuft_form(bm_area area, uint32_t layer, uint32_t tuft, bm_tuft_form* out) {
    if (!area || !out) return set_err(BM_ERR_INVALID, "null argument");
    if (layer >= area->plan.n_layers || tuft >= area->plan.layers[layer].n_tufts)
        return set_err(BM_ERR_INVALID, "layer %u tuft %u out of range", layer, tuft);
    DevGuard g(area->ctx->device);
    *out = bm_tuft_form{};
    const FusedTuft& FT = area->fused.t[layer][tuft];
    const bm_layer_plan& L = area->plan.layers[layer];
    if (area->exec_path != BM_PATH_FUSED || !FT.ok) return BM_OK;
    // The status words reflect the sources and flags as of the last write.
    run_pending_verifies(area, area->stream());
    unsigned int status = 0;
    CU(cudaMemcpyAsync(&status, &area->ctl->tuft_status[layer * BM_MAX_TUFTS + tuft], sizeof status,
                       cudaMemcpyDeviceToHost, area->stream()));
    CU(cudaStreamSynchronize(area->stream()));
    out->fused = 1;
    out->tiled = FT.tiled ? 1 : 0;
    out->consumer = consumer_shape(FT, L.tufts[tuft].syns_per_tft, L.tufts[tuft].syns_per_den,
                                   L.kind == BM_LYR_PYRAMIDAL);
    out->sources_outside = (status & kTuftSrcOutsideTile) ? 1 : 0;
    out->flags_foreign = (status & kTuftFlagsForeign) ? 1 : 0;
    if (FT.tiled) {
        out->tile_w = FT.tile_w;
        out->tile_h = FT.tile_h;
        out->stages = FT.nst;
        out->grid = FT.grid;
        out->smem = FT.smem;
        out->footprint_tma = FT.fp_tma ? 1 : 0;
    }
    return BM_OK;
}

int bm_area_get_cycle(bm_area area, uint64_t* out) {
    if (!area || !out) return set_err(BM_ERR_INVALID, "null argument");
    *out = area->host_cycle;
    return BM_OK;
}

int bm_area_set_cycle(bm_area area, uint64_t cycle) {
    if (!area) return set_err(BM_ERR_INVALID, "null area");
    DevGuard g(area->ctx->device);
    // Only the counter: the error bits and the tufts' verification status stay.
    unsigned long long c = cycle;
    CU(cudaMemcpyAsync(&area->ctl->cycle, &c, sizeof c, cudaMemcpyHostToDevice, area->stream()));
    CU(cudaStreamSynchronize(area->stream()));
    area->host_cycle = cycle;
    return BM_OK;
}

int bm_area_front_steps(bm_area area, uint32_t* n) {
    if (!area || !n) return set_err(BM_ERR_INVALID, "null argument");
    *n = area->front_active() ? (uint32_t)area->front_n : 0u;
    return BM_OK;
}

int bm_area_side_steps(bm_area area, uint32_t* n) {
    if (!area || !n) return set_err(BM_ERR_INVALID, "null argument");
    uint32_t c = 0;
    for (uint8_t x : area->step_side) c += x;
    *n = c;
    return BM_OK;
}

int bm_area_slab_ptr(bm_area area, void** out) {
    if (!area || !out) return set_err(BM_ERR_INVALID, "null argument");
    *out = area->slab;
    return BM_OK;
}

int bm_area_set_profiling(bm_area area, int on) {
    if (!area) return set_err(BM_ERR_INVALID, "null area");
    area->profiling = on != 0;
    return BM_OK;
}

int bm_area_get_profile(bm_area area, uint32_t n_max, const char** names, uint64_t* launches, double* ms,
                        uint32_t* n_out) {
    if (!area || !n_out) return set_err(BM_ERR_INVALID, "null argument");
    DevGuard g(area->ctx->device);
    area->drain_profile();
    uint32_t n = 0;
    for (int k = 0; k < K_COUNT && n < n_max; k++) {
        if (!area->prof_launches[k]) continue;
        if (names) names[n] = kKindNames[k];
        if (launches) launches[n] = area->prof_launches[k];
        if (ms) ms[n] = area->prof_ms[k];
        n++;
    }
    *n_out = n;
    return BM_OK;
}

int bm_area_reset_profile(bm_area area) {
    if (!area) return set_err(BM_ERR_INVALID, "null area");
    DevGuard g(area->ctx->device);
    area->drain_profile();
    for (int k = 0; k < K_COUNT; k++) { area->prof_launches[k] = 0; area->prof_ms[k] = 0; }
    return BM_OK;
}

int bm_area_launches_per_cycle(bm_area area, uint32_t* out) {
    if (!area || !out) return set_err(BM_ERR_INVALID, "null argument");
    *out = area->launches;
    return BM_OK;
}

}  // extern "C"
