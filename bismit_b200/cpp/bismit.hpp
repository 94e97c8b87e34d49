// bismit.hpp -- the host side of bismit's cortical cycle in C++, above the C
// ABI (include/bismit_b200.h). Header only; link libbismit_b200.so.
//
// It mirrors the Rust surface this path sits behind, with the same builder
// names and argument meanings:
//   layer maps     LayerMapScheme / LayerScheme / CellScheme / TuftScheme /
//                  TuftSourceLayer / AxonDomain      (src/map/scheme/*.rs)
//   areas          AreaScheme / AreaSchemeList        (src/map/scheme/area.rs:22-198)
//   settings       CorticalAreaSettings               (src/cortex/cortical_area.rs:253-338)
//   the cortex     Cortex::builder(lmaps, areas).ca_settings(s).build(),
//                  Cortex::cycle, CorticalArea I/O    (src/cortex/cortex.rs:46-201,
//                                                      src/cortex/cortical_area.rs:343-1321)
// Input-layer sources resolve as LayerInfo::new does
// (src/map/layer_info.rs:14-100,142-215). Errors are CmnError exceptions
// carrying the C status code and message (src/cmn/error.rs).
#pragma once

#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <optional>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/bismit_b200.h"

namespace bismit {

// ------------------------------------------------------------------ errors --

struct CmnError : std::runtime_error {
    int code;
    CmnError(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

inline void check(int rc) {
    if (rc != BM_OK) throw CmnError(rc, std::string("bismit_b200: ") + bm_last_error());
}

inline void invalid(const std::string& msg) { throw CmnError(BM_ERR_INVALID, msg); }

// ------------------------------------------------------------- map pieces --

// LayerTags bits (src/map/layer_tags.rs:121-150, high word).
namespace LayerTags {
constexpr uint64_t DEFAULT = 0, PRIMARY = BM_TAG_PRIMARY, SPATIAL = BM_TAG_SPATIAL, TEMPORAL = BM_TAG_TEMPORAL,
                   FOCUS = BM_TAG_FOCUS, MOTOR = BM_TAG_MOTOR, UNUSED = BM_TAG_UNUSED, INPUT = BM_TAG_INPUT,
                   OUTPUT = BM_TAG_OUTPUT, PSAL = BM_TAG_PRIMARY | BM_TAG_SPATIAL,
                   PTAL = BM_TAG_PRIMARY | BM_TAG_TEMPORAL;
}

// Axon tags (src/map/axon_tags.rs:55-57).
inline const char* const THAL_SP = "thal_sp";
inline const char* const THAL_NSP = "thal_nsp";
inline const char* const THAL_ASC = "thal_asc";

enum class AxonTopology : uint32_t { Spatial = BM_TOPO_SPATIAL, Nonspatial = BM_TOPO_NONSPATIAL, None = BM_TOPO_NONE };
enum class InputTrack { Afferent, Efferent, Other };
enum class LayerMapKind { Cortical, Subcortical };

struct AxonSig {
    InputTrack track;
    std::set<std::string> tags;
};

// AxonDomain::{Local, input(..), output(..)} (src/map/mod.rs).
struct AxonDomain {
    uint32_t kind = BM_DOM_LOCAL;
    std::vector<AxonSig> sigs;

    static AxonDomain Local() { return AxonDomain{}; }
    static AxonDomain input(const std::vector<std::pair<InputTrack, std::vector<std::string>>>& s) {
        AxonDomain d;
        d.kind = BM_DOM_INPUT;
        for (auto& [track, tags] : s) d.sigs.push_back({track, std::set<std::string>(tags.begin(), tags.end())});
        return d;
    }
    static AxonDomain output(const std::vector<std::string>& tags) {
        AxonDomain d;
        d.kind = BM_DOM_OUTPUT;
        d.sigs.push_back({InputTrack::Other, std::set<std::string>(tags.begin(), tags.end())});
        return d;
    }
};

// TuftSourceLayer::define(name).syn_reach(r).prevalence(p) (src/map/scheme/cell.rs:6-92).
struct TuftSourceLayer {
    std::string name;
    std::optional<int32_t> reach;
    std::optional<uint32_t> prevalence_;

    static TuftSourceLayer define(const std::string& n) { return TuftSourceLayer{n, {}, {}}; }
    TuftSourceLayer syn_reach(int32_t r) const { auto c = *this; c.reach = r; return c; }
    TuftSourceLayer prevalence(uint32_t p) const { auto c = *this; c.prevalence_ = p; return c; }
    TuftSourceLayer build() const {
        if (!reach || !prevalence_) invalid("TuftSourceLayerDefinition::build: syn_reach and prevalence are required");
        if (*prevalence_ < 1) invalid("Tuft source layer definitions must have a prevalence of at least one.");
        return *this;
    }
};

// TuftScheme builder (src/map/scheme/cell.rs:95-263).
struct TuftScheme {
    std::optional<uint32_t> den_class, den_kind, syns;
    uint32_t dens = 1, mad_l2 = 0;
    std::optional<int64_t> thresh;
    std::vector<TuftSourceLayer> srcs;

    static TuftScheme basal() { TuftScheme t; t.den_class = BM_DEN_BASAL; return t; }
    static TuftScheme apical() { TuftScheme t; t.den_class = BM_DEN_APICAL; return t; }
    TuftScheme proximal() const { auto c = *this; c.den_kind = BM_DEN_PROXIMAL; return c; }
    TuftScheme distal() const { auto c = *this; c.den_kind = BM_DEN_DISTAL; return c; }
    TuftScheme dens_per_tft(uint32_t n) const { auto c = *this; c.dens = n; return c; }
    TuftScheme syns_per_den(uint32_t n) const { auto c = *this; c.syns = n; return c; }
    TuftScheme max_active_dens_l2(uint32_t n) const { auto c = *this; c.mad_l2 = n; return c; }
    TuftScheme thresh_init(int64_t n) const { auto c = *this; c.thresh = n; return c; }
    TuftScheme src_lyr(const TuftSourceLayer& s) const { auto c = *this; c.srcs.push_back(s.build()); return c; }
};

// ControlCellKind variants on this path (src/map/mod.rs).
struct ControlCellKind {
    uint32_t kind;
    std::string host_lyr_name;
    uint32_t field_radius = 0;

    static ControlCellKind InhibitoryBasketSurround(const std::string& host, uint32_t radius) {
        return {BM_LYR_CTRL_INHIB_BASKET, host, radius};
    }
    static ControlCellKind PyrOutputter(const std::string& host) { return {BM_LYR_CTRL_PYR_OUTPUT, host, 0}; }
    static ControlCellKind IntraColumnInhib(const std::string& host) { return {BM_LYR_CTRL_INTRA_COLUMN, host, 0}; }
    static ControlCellKind ActivitySmoother(const std::string& host, uint32_t radius) {
        return {BM_LYR_CTRL_SMOOTHER, host, radius};
    }
};

// CellScheme::{spiny_stellate, pyramidal, control} (src/map/scheme/cell.rs).
struct CellScheme {
    uint32_t kind;
    std::vector<TuftScheme> tfts;
    std::optional<ControlCellKind> ctrl;
    uint32_t exe_order = 0;

    static CellScheme spiny_stellate() { return CellScheme{BM_LYR_SPINY_STELLATE, {}, {}, 0}; }
    static CellScheme pyramidal() { return CellScheme{BM_LYR_PYRAMIDAL, {}, {}, 0}; }
    static CellScheme control(const ControlCellKind& k, uint32_t exe_order) {
        return CellScheme{k.kind, {}, k, exe_order};
    }
    CellScheme tft(const TuftScheme& t) const {
        if (!t.den_class || !t.den_kind || !t.syns) invalid("TuftScheme::build: class, kind and syns_per_den are required");
        auto c = *this;
        c.tfts.push_back(t);
        return c;
    }
};

// LayerScheme::define(name)... (src/map/scheme/layer.rs:42-130).
struct LayerScheme {
    std::string name;
    std::optional<int32_t> depth_;
    uint64_t tags_ = LayerTags::DEFAULT;
    uint32_t kind = BM_LYR_AXONAL;
    AxonTopology topology = AxonTopology::Spatial;
    AxonDomain domain;
    std::optional<CellScheme> cell;

    static LayerScheme define(const std::string& n) { LayerScheme l; l.name = n; return l; }
    LayerScheme depth(int32_t d) const { auto c = *this; c.depth_ = d; return c; }
    LayerScheme tags(uint64_t t) const { auto c = *this; c.tags_ = t; return c; }
    LayerScheme axonal(AxonTopology t) const { auto c = *this; c.kind = BM_LYR_AXONAL; c.topology = t; return c; }
    LayerScheme axon_domain(const AxonDomain& d) const { auto c = *this; c.domain = d; return c; }
    LayerScheme cellular(const CellScheme& cs) const { auto c = *this; c.cell = cs; c.kind = cs.kind; return c; }
};

struct LayerMapScheme {
    std::string name;
    LayerMapKind kind = LayerMapKind::Cortical;
    std::vector<LayerScheme> layers;

    LayerMapScheme(std::string n, LayerMapKind k) : name(std::move(n)), kind(k) {}
    LayerMapScheme& layer(const LayerScheme& l) {
        layers.push_back(l);
        return *this;
    }
    // Output layers whose axon tags include all of `tags`.
    std::vector<const LayerScheme*> output_layers_with_axon_tags(const std::set<std::string>& tags) const {
        std::vector<const LayerScheme*> out;
        for (const auto& l : layers) {
            if (l.domain.kind != BM_DOM_OUTPUT) continue;
            for (const auto& s : l.domain.sigs) {
                bool all = true;
                for (const auto& t : tags) all = all && s.tags.count(t);
                if (all) {
                    out.push_back(&l);
                    break;
                }
            }
        }
        return out;
    }
};

struct LayerMapSchemeList {
    std::map<std::string, LayerMapScheme> maps;
    LayerMapSchemeList& lmap(const LayerMapScheme& m) {
        maps.erase(m.name);
        maps.emplace(m.name, m);
        return *this;
    }
    const LayerMapScheme& operator[](const std::string& n) const {
        auto it = maps.find(n);
        if (it == maps.end()) invalid("no layer map named '" + n + "'");
        return it->second;
    }
};

// AreaScheme::new(name, layer_map_name, side) (src/map/scheme/area.rs:22-198).
// FilterScheme::new(filter_name, cl_file_name) (src/map/scheme/filter.rs:3-40):
// one filter of an input filter chain, named by its kernel. The built-in
// filter is "retina" (cl/filters.cl:34-100); a kernel from a custom OpenCL
// file has no counterpart here.
struct FilterScheme {
    std::string filter_name;
    uint32_t kind = 0;
    FilterScheme(const std::string& name, const char* cl_file_name = nullptr) : filter_name(name) {
        if (name != "retina") invalid("unknown filter '" + name + "' (built in: retina)");
        if (cl_file_name) invalid("filter '" + name + "': kernels from custom OpenCL files are not supported");
        kind = BM_FILTER_RETINA;
    }
};

struct FilterChain {
    AxonSig sig;
    std::vector<FilterScheme> filters;
};

struct AreaScheme {
    std::string name, layer_map_name;
    uint32_t v_size, u_size;
    std::vector<std::string> eff, aff, other;
    std::vector<FilterChain> chains;

    AreaScheme(std::string n, std::string lm, uint32_t side)
        : name(std::move(n)), layer_map_name(std::move(lm)), v_size(side), u_size(side) {}
    static AreaScheme irregular(const std::string& n, const std::string& lm, uint32_t v, uint32_t u) {
        AreaScheme a(n, lm, v);
        a.u_size = u;
        return a;
    }
    AreaScheme eff_areas(std::vector<std::string> v) const { auto c = *this; c.eff = std::move(v); return c; }
    AreaScheme aff_areas(std::vector<std::string> v) const { auto c = *this; c.aff = std::move(v); return c; }
    AreaScheme other_areas(std::vector<std::string> v) const { auto c = *this; c.other = std::move(v); return c; }
    // AreaScheme::filter_chain (src/map/scheme/area.rs:70-85): frames of the
    // source matched by the input signature (track, tags) pass through the
    // filters in order.
    AreaScheme filter_chain(InputTrack track, const std::vector<std::string>& tags,
                            std::vector<FilterScheme> filters) const {
        if (filters.size() > BM_MAX_FILTERS) invalid("more than " + std::to_string(BM_MAX_FILTERS) + " filters in one chain");
        auto c = *this;
        c.chains.push_back({{track, std::set<std::string>(tags.begin(), tags.end())}, std::move(filters)});
        return c;
    }
};

struct AreaSchemeList {
    std::vector<AreaScheme> areas;
    AreaSchemeList& area(const AreaScheme& a) {
        areas.push_back(a);
        return *this;
    }
    const AreaScheme& by_name(const std::string& n) const {
        for (const auto& a : areas)
            if (a.name == n) return a;
        invalid("no area named '" + n + "'");
        throw;   // unreachable
    }
    uint32_t area_id(const std::string& n) const {
        for (uint32_t i = 0; i < areas.size(); i++)
            if (areas[i].name == n) return i;
        invalid("no area named '" + n + "'");
        return 0;
    }
};

// CorticalAreaSettings (src/cortex/cortical_area.rs:253-338).
struct CorticalAreaSettings {
    uint32_t bits = 0, init_flags = 0, exec_path = BM_PATH_FUSED;

    CorticalAreaSettings with(uint32_t b) const { auto c = *this; c.bits |= b; return c; }
    CorticalAreaSettings bypass_inhib() const { return with(BM_SET_BYPASS_INHIB); }
    CorticalAreaSettings bypass_filters() const { return with(BM_SET_BYPASS_FILTERS); }
    CorticalAreaSettings disable_pyrs() const { return with(BM_SET_DISABLE_PYRS); }
    CorticalAreaSettings disable_sscs() const { return with(BM_SET_DISABLE_SSCS); }
    CorticalAreaSettings disable_mcols() const { return with(BM_SET_DISABLE_MCOLS); }
    CorticalAreaSettings disable_regrowth() const { return with(BM_SET_DISABLE_REGROWTH); }
    CorticalAreaSettings disable_learning() const { return with(BM_SET_DISABLE_LEARNING); }
    CorticalAreaSettings strengths_start_at_zero() const {
        auto c = *this;
        c.init_flags |= BM_INIT_STRENGTH_ZERO;
        return c;
    }
    // One kernel per reference stage instead of the fused kernels.
    CorticalAreaSettings plain_kernels() const {
        auto c = *this;
        c.exec_path = BM_PATH_PLAIN;
        return c;
    }
};

// -------------------------------------------------------------- resolution --

struct SourceLayer {
    std::string area, layer;
    uint32_t v_size, u_size, depth;
    AxonTopology topology;
};

// matching_source_layers (src/map/layer_info.rs:14-100): the source layers
// feeding an input layer with signatures `sigs`, in slice order.
inline std::vector<SourceLayer> source_list(const AreaScheme& a, const AreaSchemeList& areas,
                                            const LayerMapSchemeList& lmaps, const std::vector<AxonSig>& sigs) {
    std::vector<SourceLayer> out;
    for (const auto& sig : sigs) {
        const auto& cands = sig.track == InputTrack::Afferent ? a.eff : sig.track == InputTrack::Efferent ? a.aff : a.other;
        for (const auto& an : cands) {
            const AreaScheme& src = areas.by_name(an);
            for (const LayerScheme* l : lmaps[src.layer_map_name].output_layers_with_axon_tags(sig.tags)) {
                const uint32_t depth = l->depth_ ? (uint32_t)*l->depth_ : 1;   // DEFAULT_OUTPUT_LAYER_DEPTH
                const AxonTopology topo = l->kind == BM_LYR_AXONAL ? l->topology : AxonTopology::Spatial;
                out.push_back({an, l->name, src.v_size, src.u_size, depth, topo});
            }
        }
    }
    return out;
}

// Resolves cortical area `name` of `areas` into the C descriptor.
inline bm_area_desc area_desc(const std::string& name, const LayerMapSchemeList& lmaps, const AreaSchemeList& areas,
                              const CorticalAreaSettings& settings) {
    const AreaScheme& a = areas.by_name(name);
    const LayerMapScheme& lm = lmaps[a.layer_map_name];
    if (lm.kind != LayerMapKind::Cortical) invalid("area '" + name + "' has a subcortical layer map");
    if (lm.layers.size() > BM_MAX_LAYERS) invalid("too many layers");
    bm_area_desc d;
    std::memset(&d, 0, sizeof d);
    d.area_id = areas.area_id(name);
    d.v_size = a.v_size;
    d.u_size = a.u_size;
    d.n_layers = (uint32_t)lm.layers.size();
    d.settings = settings.bits;
    d.init_flags = settings.init_flags;
    d.exec_path = settings.exec_path;
    std::map<std::string, int32_t> idx;
    for (size_t i = 0; i < lm.layers.size(); i++) idx[lm.layers[i].name] = (int32_t)i;
    for (size_t i = 0; i < lm.layers.size(); i++) {
        const LayerScheme& ls = lm.layers[i];
        bm_layer_desc& L = d.layers[i];
        if (ls.name.size() >= BM_NAME_LEN) invalid("layer name too long: '" + ls.name + "'");
        std::memcpy(L.name, ls.name.c_str(), ls.name.size() + 1);
        L.tags = ls.tags_;
        L.kind = ls.kind;
        L.depth = ls.depth_ ? *ls.depth_ : -1;
        L.axon_topology = (uint32_t)ls.topology;
        L.axon_domain = ls.domain.kind;
        L.host_layer_idx = -1;
        if (ls.domain.kind == BM_DOM_INPUT) {
            auto srcs = source_list(a, areas, lmaps, ls.domain.sigs);
            if (srcs.size() > BM_MAX_IO) invalid("too many input sources");
            L.n_input_srcs = (uint32_t)srcs.size();
            for (size_t k = 0; k < srcs.size(); k++)
                L.input_srcs[k] = {srcs[k].v_size, srcs[k].u_size, srcs[k].depth, (uint32_t)srcs[k].topology};
        }
        if (ls.cell && ls.cell->ctrl) {
            auto it = idx.find(ls.cell->ctrl->host_lyr_name);
            if (it == idx.end()) invalid("control host layer '" + ls.cell->ctrl->host_lyr_name + "' not in the layer map");
            L.host_layer_idx = it->second;
            L.field_radius = ls.cell->ctrl->field_radius;
            L.exe_order = ls.cell->exe_order;
        } else if (ls.cell) {
            if (ls.cell->tfts.size() > BM_MAX_TUFTS) invalid("too many tufts");
            L.n_tufts = (uint32_t)ls.cell->tfts.size();
            for (size_t t = 0; t < ls.cell->tfts.size(); t++) {
                const TuftScheme& ts = ls.cell->tfts[t];
                bm_tuft_desc& T = L.tufts[t];
                T.den_class = *ts.den_class;
                T.den_kind = *ts.den_kind;
                T.dens_per_tft = ts.dens;
                T.syns_per_den = *ts.syns;
                T.max_active_dens_l2 = ts.mad_l2;
                T.thresh_init = ts.thresh ? *ts.thresh : -1;
                if (ts.srcs.size() > BM_MAX_SRC_LAYERS) invalid("too many tuft sources");
                T.n_src = (uint32_t)ts.srcs.size();
                for (size_t k = 0; k < ts.srcs.size(); k++) {
                    auto it = idx.find(ts.srcs[k].name);
                    if (it == idx.end()) invalid("tuft source layer '" + ts.srcs[k].name + "' not in the layer map");
                    T.src[k] = {it->second, *ts.srcs[k].reach, *ts.srcs[k].prevalence_};
                }
            }
        }
    }
    // Each filter chain goes to the one source whose input signature it names
    // (AxonSpace::new, src/cortex/axon_space.rs:340-345, with
    // LayerMap::src_layer_info_by_sig, src/map/layer_map.rs:242-261).
    for (const FilterChain& ch : a.chains) {
        std::vector<std::pair<size_t, size_t>> hits;
        for (size_t i = 0; i < lm.layers.size(); i++) {
            const LayerScheme& ls = lm.layers[i];
            if (ls.domain.kind != BM_DOM_INPUT) continue;
            size_t k = 0;
            for (const AxonSig& sig : ls.domain.sigs) {
                const size_t n = source_list(a, areas, lmaps, {sig}).size();
                if (sig.track == ch.sig.track && sig.tags == ch.sig.tags)
                    for (size_t j = 0; j < n; j++) hits.push_back({i, k + j});
                k += n;
            }
        }
        if (hits.empty()) invalid("Unable to find a layer within the area map matching the axon domain specified by a filter chain scheme.");
        if (hits.size() > 1) invalid("Duplicate axon signatures found within the layer map for area '" + name + "'.");
        bm_input_src_desc& S = d.layers[hits[0].first].input_srcs[hits[0].second];
        if (S.n_filters) invalid("two filter chains for one source");
        S.n_filters = (uint32_t)ch.filters.size();
        for (size_t j = 0; j < ch.filters.size(); j++) S.filters[j] = ch.filters[j].kind;
    }
    return d;
}

// A tract between two areas of a cortex (thalamic routing).
struct Tract {
    uint32_t src_area, src_output, dst_area, dst_input;
    uint64_t dst_offset, length;
};

// An input no area of the cortex feeds: written by the caller.
struct ExternalInput {
    std::string area;
    uint32_t input;
    uint64_t offset, length;
    std::string src_area, src_layer;
};

// ---------------------------------------------------------------- runtime --

// SamplerKind (src/cortex/cortical_area.rs:61-90): the buffer a sampler reads.
enum class SamplerKind : uint32_t {
    Axons = BM_BUF_AXON_STATES,
    SomaStates = BM_BUF_CEL_STATES,
    SomaEnergies = BM_BUF_CEL_ENERGIES,
    SomaActivities = BM_BUF_CEL_ACTIVITIES,
    SomaFlagSets = BM_BUF_CEL_FLAG_SETS,
    TuftStates = BM_BUF_TFT_STATES,
    TuftBestDenIds = BM_BUF_TFT_BEST_DEN_IDS,
    TuftBestDenStatesRaw = BM_BUF_TFT_BEST_DEN_STATES_RAW,
    TuftBestDenStates = BM_BUF_TFT_BEST_DEN_STATES,
    TuftPrevStates = BM_BUF_TFT_PREV_STATES,
    TuftPrevBestDenIds = BM_BUF_TFT_PREV_BEST_DEN_IDS,
    TuftPrevBestDenStatesRaw = BM_BUF_TFT_PREV_BEST_DEN_STATES_RAW,
    TuftPrevBestDenStates = BM_BUF_TFT_PREV_BEST_DEN_STATES,
    DenStates = BM_BUF_DEN_STATES,
    DenStatesRaw = BM_BUF_DEN_STATES_RAW,
    DenEnergies = BM_BUF_DEN_ENERGIES,
    DenActivities = BM_BUF_DEN_ACTIVITIES,
    DenThresholds = BM_BUF_DEN_THRESHOLDS,
    SynStates = BM_BUF_SYN_STATES,
    SynStrengths = BM_BUF_SYN_STRENGTHS,
    SynSrcSlcIds = BM_BUF_SYN_SRC_SLC_IDS,
    SynSrcColVOffs = BM_BUF_SYN_SRC_COL_V_OFFS,
    SynSrcColUOffs = BM_BUF_SYN_SRC_COL_U_OFFS,
    SynFlagSets = BM_BUF_SYN_FLAG_SETS,
};

// The receiving end of a sampler (TractReceiver, src/subcortex/tract_channel.rs:
// 535-548). Owned by its area, which destroys it first.
class Sampler {
   public:
    explicit Sampler(bm_sampler h) : h_(h) { check(bm_sampler_len(h_, &len_)); }
    ~Sampler() {
        if (h_) bm_sampler_destroy(h_);
    }
    Sampler(const Sampler&) = delete;
    Sampler& operator=(const Sampler&) = delete;

    uint64_t len() const { return len_; }
    // TractReceiver::recv: true with the unread frame (and the cycle whose end
    // state it holds), or false when there is none and wait_for_frame is off.
    bool recv(bool wait_for_frame, std::vector<uint8_t>& frame, uint64_t* cycle = nullptr) {
        frame.resize(len_);
        int got = 0;
        uint64_t c = 0;
        check(bm_sampler_recv(h_, wait_for_frame ? 1 : 0, frame.data(), len_, &c, &got));
        if (cycle) *cycle = c;
        return got != 0;
    }
    // TractReceiver::set_backpressure: returns the prior state.
    bool set_backpressure(bool on) {
        int prior = 0;
        check(bm_sampler_set_backpressure(h_, on ? 1 : 0, &prior));
        return prior != 0;
    }
    void set_timeout(uint32_t ms) { check(bm_sampler_set_timeout(h_, ms)); }

   private:
    bm_sampler h_ = nullptr;
    uint64_t len_ = 0;
};

class CorticalArea {
   public:
    CorticalArea(bm_ctx ctx, const bm_area_desc& desc, uint64_t seed, std::string name)
        : name_(std::move(name)), desc_(desc) {
        check(bm_area_create(ctx, &desc_, seed, &h_));
        check(bm_area_get_plan(h_, &plan_));
    }
    ~CorticalArea() {
        samplers_.clear();
        if (h_) bm_area_destroy(h_);
    }
    CorticalArea(const CorticalArea&) = delete;
    CorticalArea& operator=(const CorticalArea&) = delete;

    const std::string& name() const { return name_; }
    const bm_area_plan& plan() const { return plan_; }
    bm_area handle() const { return h_; }

    // AxonSpace::intake (src/cortex/axon_space.rs:509-588).
    void write_input(const std::vector<uint8_t>& frame, uint32_t input = 0) {
        check(bm_area_write_input(h_, input, frame.data(), frame.size()));
    }
    // CorticalArea::cycle (src/cortex/cortical_area.rs:716-789).
    void cycle(uint32_t n = 1) { check(bm_area_cycle(h_, n)); }
    // AxonSpace::output (src/cortex/axon_space.rs:594-629).
    std::vector<uint8_t> read_output(uint32_t output = 0) const {
        std::vector<uint8_t> out(plan_.outputs[output].len);
        check(bm_area_read_output(h_, output, out.data(), out.size()));
        return out;
    }
    std::vector<uint8_t> read(uint32_t buf_kind, uint32_t layer, uint64_t offset, uint64_t len) const {
        std::vector<uint8_t> out(len);
        check(bm_area_read(h_, buf_kind, layer, offset, out.data(), len));
        return out;
    }
    void write(uint32_t buf_kind, uint32_t layer, uint64_t offset, const std::vector<uint8_t>& data) {
        check(bm_area_write(h_, buf_kind, layer, offset, data.data(), data.size()));
    }
    std::vector<uint8_t> read_slab() const {
        std::vector<uint8_t> out(plan_.slab_bytes);
        check(bm_area_read_slab(h_, out.data(), out.size()));
        return out;
    }
    void write_slab(const std::vector<uint8_t>& s) { check(bm_area_write_slab(h_, s.data(), s.size())); }
    uint64_t cycle_count() const {
        uint64_t c = 0;
        check(bm_area_get_cycle(h_, &c));
        return c;
    }
    void set_cycle(uint64_t c) { check(bm_area_set_cycle(h_, c)); }

    // CorticalArea::sampler (src/cortex/cortical_area.rs:1017-1284): a
    // sampler over `kind` of data layer `layer` (for Axons, BM_ALL_LAYERS
    // samples every axon of the area).
    Sampler& sampler(SamplerKind kind, uint32_t layer, bool backpressure = false) {
        bm_sampler h = nullptr;
        check(bm_sampler_create(h_, (uint32_t)kind, layer, backpressure ? 1 : 0, &h));
        samplers_.push_back(std::make_unique<Sampler>(h));
        return *samplers_.back();
    }

   private:
    std::string name_;
    bm_area_desc desc_;
    bm_area h_ = nullptr;
    bm_area_plan plan_;
    std::vector<std::unique_ptr<Sampler>> samplers_;
};

class CortexBuilder;

// When a tract delivers its source's output.
enum class TractTiming {
    PreviousCycle,   // every tract at the head of each cycle, from the previous cycle: the areas
                     // cycle together as one batch
    SameCycle,       // bismit's order (src/cortex/cortex.rs:99-119): area after area, each taking
                     // its tracts first, so a tract from an earlier area carries this cycle's output
};

// Cortex (src/cortex/cortex.rs:37-120): its cortical areas, with the thalamic
// routes between them as tracts, cycled as `timing` says.
class Cortex {
   public:
    static CortexBuilder builder(const LayerMapSchemeList& lmaps, const AreaSchemeList& areas);

    Cortex(const LayerMapSchemeList& lmaps, const AreaSchemeList& areas, const CorticalAreaSettings& settings,
           uint64_t seed, int device, TractTiming timing = TractTiming::PreviousCycle)
        : timing_(timing) {
        check(bm_ctx_create(device, 0, &ctx_));
        try {
            for (const auto& a : areas.areas) {
                if (lmaps[a.layer_map_name].kind != LayerMapKind::Cortical) continue;
                areas_.emplace_back(new CorticalArea(ctx_, area_desc(a.name, lmaps, areas, settings), seed, a.name));
            }
            route(lmaps, areas);
            if (!areas_.empty() && timing_ == TractTiming::PreviousCycle) {
                std::vector<bm_area> hs;
                for (auto& p : areas_) hs.push_back(p->handle());
                check(bm_batch_create(ctx_, hs.data(), (uint32_t)hs.size(), &batch_));
                for (const auto& t : tracts_)
                    check(bm_batch_connect(batch_, t.src_area, t.src_output, t.dst_area, t.dst_input, t.dst_offset));
            }
        } catch (...) {
            release();
            throw;
        }
    }
    ~Cortex() { release(); }
    Cortex(const Cortex&) = delete;
    Cortex& operator=(const Cortex&) = delete;

    // Cortex::cycle (src/cortex/cortex.rs:99-119).
    void cycle(uint32_t n = 1) {
        if (batch_) {
            check(bm_batch_cycle(batch_, n));
            return;
        }
        for (uint32_t c = 0; c < n; c++)
            for (uint32_t k = 0; k < areas_.size(); k++) {
                for (const auto& t : tracts_)
                    if (t.dst_area == k)
                        check(bm_area_deliver_tract(areas_[t.src_area]->handle(), t.src_output, areas_[k]->handle(),
                                                    t.dst_input, t.dst_offset));
                areas_[k]->cycle(1);
            }
    }
    TractTiming tract_timing() const { return timing_; }
    CorticalArea& area(const std::string& name) {
        for (auto& p : areas_)
            if (p->name() == name) return *p;
        invalid("no cortical area named '" + name + "'");
        throw;   // unreachable
    }
    const std::vector<Tract>& tracts() const { return tracts_; }
    const std::vector<ExternalInput>& external_inputs() const { return external_; }
    void synchronize() { check(bm_ctx_synchronize(ctx_)); }

   private:
    void route(const LayerMapSchemeList& lmaps, const AreaSchemeList& areas) {
        std::map<std::string, uint32_t> pos;
        for (uint32_t k = 0; k < areas_.size(); k++) pos[areas_[k]->name()] = k;
        for (uint32_t k = 0; k < areas_.size(); k++) {
            const AreaScheme& a = areas.by_name(areas_[k]->name());
            const LayerMapScheme& lm = lmaps[a.layer_map_name];
            const bm_area_plan& P = areas_[k]->plan();
            for (uint32_t i = 0; i < P.n_inputs; i++) {
                const LayerScheme& ls = lm.layers[P.inputs[i].layer_idx];
                uint64_t off = 0;
                for (const auto& src : source_list(a, areas, lmaps, ls.domain.sigs)) {
                    const uint64_t len = (uint64_t)src.v_size * src.u_size * src.depth;
                    auto it = pos.find(src.area);
                    if (it != pos.end()) {
                        const bm_area_plan& S = areas_[it->second]->plan();
                        const LayerMapScheme& slm = lmaps[areas.by_name(src.area).layer_map_name];
                        uint32_t li = 0;
                        while (li < slm.layers.size() && slm.layers[li].name != src.layer) li++;
                        uint32_t o = 0;
                        while (o < S.n_outputs && S.outputs[o].layer_idx != li) o++;
                        if (o == S.n_outputs || S.outputs[o].len != len) invalid("tract from " + src.area + "." + src.layer);
                        tracts_.push_back({it->second, o, k, i, off, len});
                    } else {
                        external_.push_back({areas_[k]->name(), i, off, len, src.area, src.layer});
                    }
                    off += len;
                }
            }
        }
    }
    void release() {
        if (batch_) bm_batch_destroy(batch_);
        batch_ = nullptr;
        areas_.clear();
        if (ctx_) bm_ctx_destroy(ctx_);
        ctx_ = nullptr;
    }

    TractTiming timing_;
    bm_ctx ctx_ = nullptr;
    bm_batch batch_ = nullptr;
    std::vector<std::unique_ptr<CorticalArea>> areas_;
    std::vector<Tract> tracts_;
    std::vector<ExternalInput> external_;
};

// Cortex::builder(..).ca_settings(..).build() (src/cortex/cortex.rs:158-201).
class CortexBuilder {
   public:
    CortexBuilder(LayerMapSchemeList lmaps, AreaSchemeList areas) : lmaps_(std::move(lmaps)), areas_(std::move(areas)) {}
    CortexBuilder& ca_settings(const CorticalAreaSettings& s) {
        settings_ = s;
        return *this;
    }
    CortexBuilder& seed(uint64_t s) {
        seed_ = s;
        return *this;
    }
    CortexBuilder& device(int d) {
        device_ = d;
        return *this;
    }
    CortexBuilder& tract_timing(TractTiming t) {
        timing_ = t;
        return *this;
    }
    std::unique_ptr<Cortex> build() const {
        return std::make_unique<Cortex>(lmaps_, areas_, settings_, seed_, device_, timing_);
    }

   private:
    LayerMapSchemeList lmaps_;
    AreaSchemeList areas_;
    CorticalAreaSettings settings_ = CorticalAreaSettings().disable_regrowth();
    uint64_t seed_ = 0;
    int device_ = 0;
    TractTiming timing_ = TractTiming::PreviousCycle;
};

inline CortexBuilder Cortex::builder(const LayerMapSchemeList& lmaps, const AreaSchemeList& areas) {
    return CortexBuilder(lmaps, areas);
}

}  // namespace bismit
