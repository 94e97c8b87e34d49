// bm_layout.cpp -- resolves an area scheme (bm_area_desc) into the plan of
// index spaces and buffer offsets the kernels use (bm_area_plan).
//
// Restates the host-side map logic of bismit:
//   LayerMap::new / LayerInfo::new     src/map/layer_map.rs:66-100, src/map/layer_info.rs:116-300
//   SliceMap::new                      src/map/slice_map.rs:26-156
//   SliceDims::new, calc_scale         src/cmn/slice_dims.rs:20-121, :201-224
//   AreaMap::cel_src_slc_id_rchs       src/map/area_map.rs:139-162
//   SynSrcSlices::new, gen_syn_offs    src/map/syn_src.rs:390-446, :47-149
//   Synapses/Dendrites/Tufts index spaces
//                                      src/cortex/synapses.rs:160-199,
//                                      src/cortex/dendrites.rs:55-75, src/cortex/tufts.rs:85-101
//   role ordering                      src/cortex/cortical_area.rs:31,601-613
#include "bm_layout.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <vector>

namespace bm {

namespace {

struct Fail {
    std::string msg;
    int code = BM_ERR_INVALID;
};

[[noreturn]] void fail(const char* fmt, ...) __attribute__((format(printf, 1, 2)));
void fail(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    throw Fail{buf, BM_ERR_INVALID};
}

// calc_scale, src/cmn/slice_dims.rs:201-224.
uint32_t calc_scale(uint32_t src_dim, uint32_t tar_dim) {
    uint64_t src = (uint64_t)src_dim * 1024, tar = (uint64_t)tar_dim * 1024;
    if (tar == 0) fail("Target area dimension cannot be zero.");
    uint64_t incr = tar < 16 ? 1 : tar / 16;
    uint64_t s = src / incr;
    if (s == 0) fail("Source area dimension cannot be zero.");
    if (s > 255) fail("Source area cannot have a dimension more than 16 times target area dimension.");
    return (uint32_t)s;
}

struct SliceDims {
    uint32_t v_size, u_size, v_scale, u_scale, v_mid, u_mid;
};

// SliceDims::new, src/cmn/slice_dims.rs:20-94.
SliceDims slice_dims(uint32_t area_v, uint32_t area_u, const bm_input_src_desc* src, uint32_t topo) {
    SliceDims d{};
    if (topo == BM_TOPO_SPATIAL || topo == BM_TOPO_NONE) {
        if (src) {
            d.v_size = src->v_size;
            d.u_size = src->u_size;
            d.v_scale = calc_scale(src->v_size, area_v);
            d.u_scale = calc_scale(src->u_size, area_u);
        } else {
            d.v_size = area_v;
            d.u_size = area_u;
            d.v_scale = 16;
            d.u_scale = 16;
        }
    } else if (topo == BM_TOPO_NONSPATIAL) {
        uint32_t v = src ? src->v_size : area_v, u = src ? src->u_size : area_u;
        if (src && (v > 255 || u > 255)) fail("Dimensions size for horizontal layers may not exceed 255.");
        d.v_size = v;
        d.u_size = u;
        d.v_mid = v / 2;
        d.u_mid = u / 2;
    } else {
        fail("unknown axon topology %u", topo);
    }
    return d;
}

// gen_syn_offs, src/map/syn_src.rs:47-149.
std::vector<std::pair<int8_t, int8_t>> gen_syn_offs(int radius, uint32_t vs, uint32_t us) {
    if (radius < 0) fail("synapse reach must be >= 0 (got %d)", radius);
    int v_rad = (radius * (int)vs) >> 4, u_rad = (radius * (int)us) >> 4;
    if (std::max(v_rad, u_rad) > 127) fail("scaled synapse reach %d exceeds 127", std::max(v_rad, u_rad));
    std::vector<std::pair<int8_t, int8_t>> out;
    for (int vo = -v_rad; vo <= v_rad; vo++) {
        int a = std::max(-v_rad, -vo - v_rad), b = std::min(v_rad, -vo + v_rad);
        int uz = (a * ((int)us << 3)) / ((int)vs << 3);
        int un = (b * ((int)us << 3)) / ((int)vs << 3) + 1;
        for (int uo = uz; uo < un; uo++) {
            if (vo > 127 || vo < -127 || uo > 127 || uo < -127)
                fail("Calculated offsets are outside valid radius range: (v_ofs: %d, u_ofs: %d).", vo, uo);
            out.push_back({(int8_t)vo, (int8_t)uo});
        }
    }
    return out;
}

uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

}  // namespace

bool offset_extent(int reach, uint32_t vs, uint32_t us, int* rv, int* ru) {
    try {
        int mv = 0, mu = 0;
        for (auto& o : gen_syn_offs(reach, vs, us)) {
            mv = std::max(mv, std::abs((int)o.first));
            mu = std::max(mu, std::abs((int)o.second));
        }
        *rv = mv;
        *ru = mu;
        return true;
    } catch (const Fail&) {
        return false;
    }
}

uint64_t rnd_key(uint64_t seed, uint32_t area, uint32_t layer, uint32_t role, uint32_t tft) {
    uint64_t bits = ((uint64_t)area << 40) ^ ((uint64_t)layer << 32) ^ ((uint64_t)role << 24) ^ ((uint64_t)tft << 16);
    return splitmix64(splitmix64(seed) + bits);
}

uint64_t grow_key(uint64_t seed, uint32_t area, uint32_t layer, uint32_t tft) {
    uint64_t k = splitmix64(seed ^ 0x67726F77ull) + (((uint64_t)area << 48) | ((uint64_t)layer << 40) | ((uint64_t)tft << 32));
    return splitmix64(k);
}

// gen_grp_centers (src/cortex/smoother.rs:11-33) with HexGroupCenters
// (src/cmn/mod.rs:809-917): six lattices of hexagonal group centers of side
// r, each grown from its start by the six moves of add_surrounds within
// [-r, dims + r), as sets (the reference's hash-set order is not kept; the
// groups of one lattice do not overlap, so no result depends on it).
void smoother_centers(int r, int v_size, int u_size, std::vector<int32_t>& out, uint32_t off[7]) {
    const int l = r + 1, s = r, ls = l + s;
    const int moves[6][2] = {{-s, ls}, {l, s}, {ls, -l}, {s, -ls}, {-l, -s}, {-ls, l}};
    const int ofs = (r + 1) / 2;
    const int starts[6][2] = {{0, ofs}, {-ofs, ofs}, {-ofs, 0}, {0, -ofs}, {ofs, -ofs}, {ofs, 0}};
    out.clear();
    for (int k = 0; k < 6; k++) {
        off[k] = (uint32_t)out.size();
        std::set<std::pair<int, int>> seen;
        std::vector<std::pair<int, int>> todo;
        auto add = [&](int v, int u) {
            if (v < -r || u < -r || v >= v_size + r || u >= u_size + r) return;
            if (seen.insert({v, u}).second) todo.push_back({v, u});
        };
        add(starts[k][0], starts[k][1]);
        while (!todo.empty()) {
            const auto c = todo.back();
            todo.pop_back();
            for (const auto& m : moves) add(c.first + m[0], c.second + m[1]);
        }
        for (const auto& c : seen) out.push_back((int32_t)(((uint32_t)(uint16_t)(int16_t)c.first << 16) |
                                                           (uint16_t)(int16_t)c.second));
    }
    off[6] = (uint32_t)out.size();
}

int resolve_area(const bm_area_desc* D, uint64_t seed, bm_area_plan* P, std::vector<TuftGrowSpec>* grow,
                 std::string* err) {
    try {
        std::memset(P, 0, sizeof *P);
        if (!D) fail("null area descriptor");
        if (D->n_layers == 0 || D->n_layers > BM_MAX_LAYERS) fail("n_layers must be 1..%d", BM_MAX_LAYERS);
        if (D->v_size == 0 || D->u_size == 0 || D->v_size > 4096 || D->u_size > 4096)
            fail("area dims must be 1..4096 (got %u x %u)", D->v_size, D->u_size);
        P->area_id = D->area_id;
        P->v_size = D->v_size;
        P->u_size = D->u_size;
        P->settings = D->settings;
        P->rnd_seed = seed;

        // ---- slices (LayerMap::new + SliceMap::new) ----
        uint32_t slc_start[BM_MAX_LAYERS], slc_count[BM_MAX_LAYERS];
        uint32_t ns = 0, axons = 0;
        // Filtered sources, resolved to inputs[] once the io ranges exist.
        struct PendingChain {
            uint32_t layer;
            bm_filter_chain_plan c;
        };
        std::vector<PendingChain> chains;
        auto add_slice = [&](uint32_t layer, const SliceDims& d) {
            if (ns >= 255) fail("more than 255 axon slices");
            P->slc_axn_idz[ns] = axons;
            P->slc_v_size[ns] = d.v_size;
            P->slc_u_size[ns] = d.u_size;
            P->slc_v_scale[ns] = d.v_scale;
            P->slc_u_scale[ns] = d.u_scale;
            P->slc_v_mid[ns] = d.v_mid;
            P->slc_u_mid[ns] = d.u_mid;
            P->slc_layer[ns] = layer;
            axons += d.v_size * d.u_size;
            ns++;
        };
        for (uint32_t l = 0; l < D->n_layers; l++) {
            const bm_layer_desc& Ld = D->layers[l];
            for (uint32_t k = 0; k < l; k++)
                if (std::strncmp(Ld.name, D->layers[k].name, BM_NAME_LEN) == 0)
                    fail("duplicate layer name '%.*s'", BM_NAME_LEN, Ld.name);
            if (Ld.kind > BM_LYR_CTRL_SMOOTHER) fail("layer %u: unknown kind %u", l, Ld.kind);
            slc_start[l] = ns;
            if (Ld.axon_domain == BM_DOM_INPUT) {
                if (Ld.kind != BM_LYR_AXONAL)
                    fail("Error assembling LayerInfo for '%.*s'. Input layers must be 'AxonTopology::Axonal'.",
                         BM_NAME_LEN, Ld.name);
                if (Ld.n_input_srcs > BM_MAX_IO) fail("layer %u: too many input sources", l);
                uint32_t frame_off = 0;
                for (uint32_t s = 0; s < Ld.n_input_srcs; s++) {
                    const bm_input_src_desc& S = Ld.input_srcs[s];
                    if (S.v_size == 0 || S.u_size == 0) fail("input source dims are zero");
                    if (S.n_filters) {
                        if (S.n_filters > BM_MAX_FILTERS) fail("layer %u source %u: more than %d filters", l, s, BM_MAX_FILTERS);
                        PendingChain pc{l, {}};
                        pc.c.frame_off = frame_off;
                        pc.c.tar_slc = ns;
                        pc.c.depth = S.depth;
                        pc.c.v_size = S.v_size;
                        pc.c.u_size = S.u_size;
                        pc.c.n_filters = S.n_filters;
                        for (uint32_t k = 0; k < S.n_filters; k++) {
                            if (S.filters[k] != BM_FILTER_RETINA)
                                fail("layer %u source %u: unknown filter %u", l, s, S.filters[k]);
                            pc.c.filters[k] = S.filters[k];
                        }
                        chains.push_back(pc);
                    }
                    if (S.axon_topology != Ld.axon_topology) {
                        if (!(S.axon_topology == BM_TOPO_SPATIAL && Ld.axon_topology == BM_TOPO_NONSPATIAL))
                            fail("SliceMap::new(): Layers may only convert from Spatial -> Nonspatial");
                        if (S.v_size > 254 || S.u_size > 254)
                            fail("Nonspatial layer sources must have dimensions less than or equal to 254v x 254u.");
                    }
                    const uint32_t axons_before = axons;
                    for (uint32_t k = 0; k < S.depth; k++)
                        add_slice(l, slice_dims(D->v_size, D->u_size, &S, Ld.axon_topology));
                    frame_off += axons - axons_before;
                }
            } else {
                uint32_t depth = Ld.depth < 0 ? 0 : (uint32_t)Ld.depth;
                for (uint32_t k = 0; k < depth; k++) add_slice(l, slice_dims(D->v_size, D->u_size, nullptr, Ld.axon_topology));
            }
            slc_count[l] = ns - slc_start[l];
        }
        P->n_slices = ns;
        P->n_axons = axons;

        // ---- data layers ----
        int data_idx[BM_MAX_LAYERS];
        uint32_t nd = 0;
        for (uint32_t l = 0; l < D->n_layers; l++) {
            data_idx[l] = -1;
            uint32_t k = D->layers[l].kind;
            if (k == BM_LYR_SPINY_STELLATE || k == BM_LYR_PYRAMIDAL) data_idx[l] = (int)nd++;
        }
        P->n_layers = nd;
        for (uint32_t l = 0; l < D->n_layers; l++) {
            if (data_idx[l] < 0) continue;
            const bm_layer_desc& Ld = D->layers[l];
            bm_layer_plan& L = P->layers[data_idx[l]];
            L.layer_id = l;
            L.kind = Ld.kind;
            L.tags = Ld.tags;
            L.depth = slc_count[l];
            if (L.depth == 0) fail("cellular layer '%.*s' has depth 0", BM_NAME_LEN, Ld.name);
            if (Ld.axon_domain == BM_DOM_INPUT) fail("cellular layers cannot be input layers");
            L.base_axn_slc = slc_start[l];
            L.axn_idz = P->slc_axn_idz[slc_start[l]];
            L.v_size = D->v_size;
            L.u_size = D->u_size;
            uint64_t cells = (uint64_t)D->v_size * D->u_size * L.depth;
            if (cells > (1u << 24)) fail("layer '%.*s': more than 2^24 cells", BM_NAME_LEN, Ld.name);
            L.cells = (uint32_t)cells;
            if (Ld.n_tufts == 0 || Ld.n_tufts > BM_MAX_TUFTS) fail("layer %u: n_tufts must be 1..%d", l, BM_MAX_TUFTS);
            if (Ld.kind == BM_LYR_SPINY_STELLATE && Ld.n_tufts != 1)
                fail("spiny stellate layers have exactly one tuft (src/cortex/spiny_stellates.rs:15,57)");
            L.n_tufts = Ld.n_tufts;
            uint64_t syn_ttl = 0, den_ttl = 0;
            bool seen_prx = false, seen_dst = false, seen_apc = false;
            for (uint32_t t = 0; t < Ld.n_tufts; t++) {
                const bm_tuft_desc& Td = Ld.tufts[t];
                bm_tuft_plan& T = L.tufts[t];
                if (Td.dens_per_tft == 0) fail("TuftDims::new: dens_per_tft must be > 0.");
                if (Td.syns_per_den == 0) fail("TuftDims::new: syns_per_den must be > 0.");
                if (Td.dens_per_tft > 256) fail("dens_per_tft > 256 does not fit the u8 best-dendrite ids");
                if (Td.syns_per_den > 4096) fail("syns_per_den > 4096 is not supported");
                if (Td.max_active_dens_l2 > 23) fail("max_active_dens_l2 > 23 is not supported");
                T.tft_id = t;
                T.den_class = Td.den_class;
                T.den_kind = Td.den_kind;
                T.dens_per_tft = Td.dens_per_tft;
                T.syns_per_den = Td.syns_per_den;
                T.syns_per_tft = Td.dens_per_tft * Td.syns_per_den;
                T.max_active_dens_l2 = Td.max_active_dens_l2;
                T.den_threshold = Td.thresh_init < 0 ? 0u : (uint32_t)Td.thresh_init;
                T.syn_idz = syn_ttl;
                T.den_idz = den_ttl;
                T.cel_idz = (uint64_t)t * L.cells;
                syn_ttl += (uint64_t)L.cells * T.syns_per_tft;
                den_ttl += (uint64_t)L.cells * T.dens_per_tft;
                if (Ld.kind == BM_LYR_PYRAMIDAL) {
                    // PyramidalLayer::new, src/cortex/pyramidals.rs:84-122.
                    if (Td.den_class == BM_DEN_BASAL && Td.den_kind == BM_DEN_PROXIMAL) {
                        if (seen_prx) fail("two basal proximal tufts");
                        seen_prx = true;
                        L.bsl_prx_tft_id = t;
                        L.enabled_tft_flags |= 1;
                    } else if (Td.den_class == BM_DEN_BASAL && Td.den_kind == BM_DEN_DISTAL) {
                        if (seen_dst) fail("two basal distal tufts");
                        seen_dst = true;
                        L.bsl_dst_tft_id = t;
                        L.enabled_tft_flags |= 2;
                    } else if (Td.den_class == BM_DEN_APICAL && Td.den_kind == BM_DEN_DISTAL) {
                        if (seen_apc) fail("two apical distal tufts");
                        seen_apc = true;
                        L.apc_dst_tft_id = t;
                        L.enabled_tft_flags |= 4;
                    } else {
                        fail("apical proximal tufts are unimplemented in bismit (src/cortex/pyramidals.rs:117)");
                    }
                }
                // ---- source pool (AreaMap::cel_src_slc_id_rchs + SynSrcSlices::new) ----
                if (Td.n_src == 0 || Td.n_src > BM_MAX_SRC_LAYERS) fail("tuft %u of layer %u: n_src must be 1..%d", t, l, BM_MAX_SRC_LAYERS);
                std::map<uint8_t, int8_t> info;        // BTreeMap<slc_id, reach> (later entries overwrite)
                std::vector<uint8_t> order;            // distinct slices in first-seen order
                for (uint32_t s = 0; s < Td.n_src; s++) {
                    const bm_src_layer_desc& S = Td.src[s];
                    if (S.layer_idx < 0 || (uint32_t)S.layer_idx >= D->n_layers) fail("source layer index out of range");
                    if (S.prevalence == 0) fail("Tuft source layer definitions must have a prevalence of at least one.");
                    if (S.syn_reach < -128 || S.syn_reach > 127) fail("syn_reach must fit an i8");
                    uint32_t sl = (uint32_t)S.layer_idx;
                    for (uint32_t p = 0; p < S.prevalence; p++)
                        for (uint32_t k = 0; k < slc_count[sl]; k++) {
                            if (T.n_src >= BM_MAX_SRC_SLICES) fail("source pool larger than %d slices", BM_MAX_SRC_SLICES);
                            T.src_slc_ids[T.n_src] = (uint8_t)(slc_start[sl] + k);
                            T.src_reaches[T.n_src] = (int8_t)S.syn_reach;
                            T.n_src++;
                        }
                    for (uint32_t k = 0; k < slc_count[sl]; k++) {
                        uint8_t sid = (uint8_t)(slc_start[sl] + k);
                        if (!info.count(sid)) order.push_back(sid);
                        info[sid] = (int8_t)S.syn_reach;
                    }
                }
                if (T.n_src == 0)
                    fail("Synapses::new(): Synapse source resolution error. Layer: '%u', tuft: '%u' has no source "
                         "layers defined.", l, t);
                std::sort(order.begin(), order.end());
                TuftGrowSpec G;
                G.data_layer = (uint32_t)data_idx[l];
                G.tft = t;
                G.key = grow_key(seed, D->area_id, l, t);
                uint64_t poss = 0;
                for (uint8_t sid : order) {
                    int reach = info[sid];
                    T.src_uniq_slc_ids[T.n_src_uniq] = sid;
                    T.src_uniq_reaches[T.n_src_uniq] = (int8_t)reach;
                    T.n_src_uniq++;
                    GrowSrc gs;
                    gs.slc = sid;
                    uint64_t poss_k;
                    if (P->slc_v_scale[sid] == 0 && P->slc_u_scale[sid] == 0) {
                        // SynSrcSliceInfo::new, Nonspatial arm (src/map/syn_src.rs:248-275).
                        if (P->slc_v_size[sid] & 1)
                            fail("Nonspatial slices must have u and v sizes evenly divisible by 2.");
                        gs.nonspatial = 1;
                        gs.rv = (int32_t)(P->slc_v_size[sid] / 2);
                        gs.ru = (int32_t)(P->slc_u_size[sid] / 2);
                        poss_k = (uint64_t)P->slc_v_size[sid] * P->slc_u_size[sid] * T.n_src;
                    } else {
                        auto offs = gen_syn_offs(reach, P->slc_v_scale[sid], P->slc_u_scale[sid]);
                        int rv = (reach * (int)P->slc_v_scale[sid]) >> 4, ru = (reach * (int)P->slc_u_scale[sid]) >> 4;
                        if (rv < -128 || rv > 127 || ru < -128 || ru > 127) fail("scaled reach out of range");
                        gs.nonspatial = 0;
                        gs.rv = rv;
                        gs.ru = ru;
                        for (auto& o : offs) { gs.offs_v.push_back(o.first); gs.offs_u.push_back(o.second); }
                        poss_k = (uint64_t)offs.size() * T.n_src;
                    }
                    if (poss != 0 && poss != poss_k)
                        fail("source slices of tuft %u of layer '%.*s' offer different numbers of offset values "
                             "(SynSrcSlices::new asserts they are equal)", t, BM_NAME_LEN, Ld.name);
                    poss = poss_k;
                    G.srcs.push_back(std::move(gs));
                }
                if (poss < T.syns_per_den)
                    fail("The cells of this slice do not have enough possible synapse source offset values "
                         "(possible: %llu, needed: %u)", (unsigned long long)poss, T.syns_per_den);
                G.saturated = poss == T.syns_per_den;
                for (uint32_t k = 0; k < T.n_src; k++) {
                    G.pool[k] = T.src_slc_ids[k];
                    uint32_t j = 0;
                    while (G.srcs[j].slc != T.src_slc_ids[k]) j++;
                    G.pool_src[k] = (uint8_t)j;
                }
                G.n_pool = T.n_src;
                if (grow) grow->push_back(std::move(G));
            }
            if (syn_ttl >= (1ull << 32)) fail("layer '%.*s' has 2^32 or more synapses (u32 index space)", BM_NAME_LEN, Ld.name);
            L.n_syns = syn_ttl;
            L.n_dens = den_ttl;
            L.n_celtfts = (uint64_t)L.cells * L.n_tufts;
        }

        // ---- control layers: ordered by (host, exe_order) (src/cortex/control_cell_layer.rs:21) ----
        for (uint32_t l = 0; l < D->n_layers; l++) {
            const bm_layer_desc& Ld = D->layers[l];
            if (Ld.kind < BM_LYR_CTRL_INHIB_BASKET) continue;
            if (Ld.host_layer_idx < 0 || (uint32_t)Ld.host_layer_idx >= D->n_layers || data_idx[Ld.host_layer_idx] < 0)
                fail("control layer '%.*s': host layer must be a cellular data layer", BM_NAME_LEN, Ld.name);
            bm_layer_plan& H = P->layers[data_idx[Ld.host_layer_idx]];
            for (uint32_t k = 0; k < H.n_ctrl; k++)
                if (H.ctrl[k].exe_order == Ld.exe_order)
                    fail("Duplicate control cell layer address / order index found for layer: %.*s (%u)",
                         BM_NAME_LEN, Ld.name, Ld.exe_order);
            if (H.n_ctrl >= BM_MAX_CTRL) fail("too many control layers on one host");
            if ((Ld.kind == BM_LYR_CTRL_INHIB_BASKET || Ld.kind == BM_LYR_CTRL_SMOOTHER) && Ld.field_radius > 127)
                fail("field_radius must be <= 127");
            bm_ctrl_plan C{};
            C.kind = Ld.kind;
            C.exe_order = Ld.exe_order;
            C.field_radius = Ld.field_radius;
            C.layer_id = l;
            uint32_t pos = H.n_ctrl;
            while (pos > 0 && H.ctrl[pos - 1].exe_order > C.exe_order) { H.ctrl[pos] = H.ctrl[pos - 1]; pos--; }
            H.ctrl[pos] = C;
            H.n_ctrl++;
        }

        // ---- io ranges ----
        for (uint32_t l = 0; l < D->n_layers; l++) {
            const bm_layer_desc& Ld = D->layers[l];
            if (slc_count[l] == 0) continue;
            bm_io_plan io{l, P->slc_axn_idz[slc_start[l]], 0};
            for (uint32_t k = 0; k < slc_count[l]; k++) io.len += P->slc_v_size[slc_start[l] + k] * P->slc_u_size[slc_start[l] + k];
            if (Ld.axon_domain == BM_DOM_INPUT) {
                if (P->n_inputs >= BM_MAX_IO) fail("too many input layers");
                P->inputs[P->n_inputs++] = io;
            } else if (Ld.axon_domain == BM_DOM_OUTPUT) {
                if (P->n_outputs >= BM_MAX_IO) fail("too many output layers");
                P->outputs[P->n_outputs++] = io;
            }
        }

        // ---- input filter chains (AxonSpace::new, src/cortex/axon_space.rs:338-412) ----
        for (const PendingChain& pc : chains) {
            bm_filter_chain_plan c = pc.c;
            c.input = UINT32_MAX;
            for (uint32_t i = 0; i < P->n_inputs; i++)
                if (P->inputs[i].layer_idx == pc.layer) c.input = i;
            if (c.input == UINT32_MAX) fail("filter chain on layer %u, which is not an input layer", pc.layer);
            if (c.depth == 0) fail("filter chain on a source of depth 0 (layer %u)", pc.layer);
            // The filter kernels run as (depth, v, u) NDRanges of 1 x 8 x 8
            // work-groups (SensoryFilter::new, src/cortex/sensory_filter.rs:
            // 47-54), which OpenCL refuses unless 8 divides v and u.
            if (c.v_size % 8 || c.u_size % 8)
                fail("filter chain on layer %u: source dims %u x %u are not multiples of 8 (1 x 8 x 8 work-groups)",
                     pc.layer, c.v_size, c.u_size);
            for (uint32_t k = 0; k < c.depth; k++)
                if (P->slc_v_size[c.tar_slc + k] != c.v_size || P->slc_u_size[c.tar_slc + k] != c.u_size)
                    fail("filter chain on layer %u: target slice %u is %u x %u, the source %u x %u", pc.layer,
                         c.tar_slc + k, P->slc_v_size[c.tar_slc + k], P->slc_u_size[c.tar_slc + k], c.v_size, c.u_size);
            // A filter that feeds another writes slice k of its output at the
            // area's axon offset of slice k (get_axn_idz with a zero base,
            // cl/filters.cl:45-47), which must stay inside that buffer.
            const uint64_t len = (uint64_t)c.depth * c.v_size * c.u_size;
            if (c.n_filters > 1)
                for (uint32_t k = 0; k < c.depth; k++)
                    if ((uint64_t)P->slc_axn_idz[k] + (uint64_t)c.v_size * c.u_size > len)
                        fail("filter chain on layer %u: an inner filter would write slice %u past its %llu-byte "
                             "buffer (axon offset %u)", pc.layer, k, (unsigned long long)len, P->slc_axn_idz[k]);
            if (P->n_filter_chains >= BM_MAX_IO) fail("more than %d filter chains", BM_MAX_IO);
            P->filter_chains[P->n_filter_chains++] = c;
        }

        // ---- cycle order by role (ROLE_ORDER, src/cortex/cortical_area.rs:31,601-613) ----
        const uint64_t roles[4] = {BM_TAG_FOCUS, BM_TAG_SPATIAL, BM_TAG_TEMPORAL, BM_TAG_MOTOR};
        bool used[BM_MAX_LAYERS] = {};
        for (uint64_t role : roles)
            for (uint32_t i = 0; i < P->n_layers; i++)
                if ((P->layers[i].tags & role) && !used[i]) {
                    used[i] = true;
                    P->cycle_order[P->n_cycle_order++] = i;
                }

        // ---- slab layout: 256-byte aligned buffers ----
        uint64_t off = 0;
        P->axon_off = off;
        off = align_up(off + P->n_axons, 256);
        for (uint32_t i = 0; i < P->n_layers; i++) {
            bm_layer_plan& L = P->layers[i];
            for (int k = 0; k < BM_BUF_COUNT; k++) { L.buf_off[k] = UINT64_MAX; L.buf_len[k] = 0; }
            auto put = [&](int k, uint64_t len) {
                L.buf_off[k] = off;
                L.buf_len[k] = len;
                off = align_up(off + len, 256);
            };
            for (int k = BM_BUF_SYN_STATES; k <= BM_BUF_SYN_FLAG_SETS; k++) put(k, L.n_syns);
            for (int k = BM_BUF_DEN_STATES_RAW; k <= BM_BUF_DEN_THRESHOLDS; k++) put(k, L.n_dens);
            if (L.kind == BM_LYR_PYRAMIDAL) {
                for (int k = BM_BUF_TFT_PREV_BEST_DEN_IDS; k <= BM_BUF_TFT_STATES; k++) put(k, L.n_celtfts);
                put(BM_BUF_CEL_STATES, L.cells);
                put(BM_BUF_CEL_FLAG_SETS, L.cells);
            }
            put(BM_BUF_CEL_ENERGIES, L.cells);
            put(BM_BUF_CEL_ACTIVITIES, L.cells);
            if (!(P->settings & BM_SET_DISABLE_REGROWTH)) put(BM_BUF_DEN_SRC_KEY0, L.n_dens);
            P->n_syns_total += L.n_syns;
        }
        for (uint32_t i = 0; i < P->n_filter_chains; i++) {
            bm_filter_chain_plan& c = P->filter_chains[i];
            for (uint32_t k = 0; k < c.n_filters; k++) {
                c.buf_off[k] = off;
                off = align_up(off + (uint64_t)c.depth * c.v_size * c.u_size, 256);
            }
        }
        P->slab_bytes = off;
        return BM_OK;
    } catch (const Fail& f) {
        if (err) *err = f.msg;
        return f.code;
    }
}

}  // namespace bm
