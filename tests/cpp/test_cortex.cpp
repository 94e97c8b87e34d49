// C++ host mirror checks, driven by tests/test_cpp_host.py.
//   test_cortex desc <dir>   writes the bm_area_desc bytes the C++ builders
//                            resolve for each case (compared with the Python
//                            mirror's), and checks the builders' error paths
//   test_cortex cycle <dir>  builds the three-area hierarchy through
//                            Cortex::builder, writes each area's grown state,
//                            cycles it on frames read from <dir>/frames.bin,
//                            and writes each area's final state (compared
//                            with the oracle run under the same tract timing)
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "bismit.hpp"

using namespace bismit;

namespace {

void external(LayerMapSchemeList& lmaps, AreaSchemeList& areas, const std::string& name, uint32_t side,
              bool nonspatial = false) {
    LayerMapScheme lm(name + "_lm", LayerMapKind::Subcortical);
    lm.layer(LayerScheme::define("ganglion").depth(1).axonal(AxonTopology::Spatial)
                 .axon_domain(AxonDomain::output({THAL_SP})));
    if (nonspatial)
        lm.layer(LayerScheme::define("ganglion_ns").depth(1).axonal(AxonTopology::Nonspatial)
                     .axon_domain(AxonDomain::output({THAL_NSP})));
    lmaps.lmap(lm);
    areas.area(AreaScheme(name, lm.name, side));
}

// The benchmark layer map (the Python configs.benchmark_area).
void benchmark_area(LayerMapSchemeList& lmaps, AreaSchemeList& areas, uint32_t side, uint32_t ssc_syns,
                    int pyr_depth, uint32_t prox_dens, uint32_t prox_syns, int prox_reach) {
    external(lmaps, areas, "v0", side);
    LayerMapScheme lm("visual", LayerMapKind::Cortical);
    lm.layer(LayerScheme::define("aff_in").axonal(AxonTopology::Spatial)
                 .axon_domain(AxonDomain::input({{InputTrack::Afferent, {THAL_SP}}})));
    lm.layer(LayerScheme::define("iv").depth(1).tags(LayerTags::PSAL).axon_domain(AxonDomain::Local())
                 .cellular(CellScheme::spiny_stellate().tft(TuftScheme::basal().proximal().syns_per_den(ssc_syns)
                     .src_lyr(TuftSourceLayer::define("aff_in").syn_reach(6).prevalence(1)))));
    lm.layer(LayerScheme::define("iv_inhib")
                 .cellular(CellScheme::control(ControlCellKind::InhibitoryBasketSurround("iv", 4), 0)));
    lm.layer(LayerScheme::define("iii").depth(pyr_depth).tags(LayerTags::PTAL)
                 .axon_domain(AxonDomain::output({THAL_SP}))
                 .cellular(CellScheme::pyramidal()
                     .tft(TuftScheme::basal().proximal().dens_per_tft(prox_dens).syns_per_den(prox_syns)
                         .src_lyr(TuftSourceLayer::define("iv").syn_reach(prox_reach).prevalence(1)))
                     .tft(TuftScheme::basal().distal().dens_per_tft(16).syns_per_den(32).max_active_dens_l2(3)
                         .src_lyr(TuftSourceLayer::define("iii").syn_reach(6).prevalence(1)))));
    lm.layer(LayerScheme::define("iii_col")
                 .cellular(CellScheme::control(ControlCellKind::IntraColumnInhib("iii"), 0)));
    lmaps.lmap(lm);
    areas.area(AreaScheme("v1", "visual", side).eff_areas({"v0"}));
}

// The mixed parity case (the Python configs.mixed_area).
void mixed_area(LayerMapSchemeList& lmaps, AreaSchemeList& areas, uint32_t side, uint32_t src_side) {
    external(lmaps, areas, "v0", src_side, true);
    LayerMapScheme lm("visual", LayerMapKind::Cortical);
    lm.layer(LayerScheme::define("aff_in").axonal(AxonTopology::Spatial)
                 .axon_domain(AxonDomain::input({{InputTrack::Afferent, {THAL_SP}}})));
    lm.layer(LayerScheme::define("ns_in").axonal(AxonTopology::Nonspatial)
                 .axon_domain(AxonDomain::input({{InputTrack::Afferent, {THAL_NSP}}})));
    lm.layer(LayerScheme::define("iv").depth(2).tags(LayerTags::PSAL)
                 .cellular(CellScheme::spiny_stellate().tft(TuftScheme::basal().proximal().syns_per_den(24).thresh_init(40)
                     .src_lyr(TuftSourceLayer::define("aff_in").syn_reach(4).prevalence(2)))));
    lm.layer(LayerScheme::define("iv_inhib")
                 .cellular(CellScheme::control(ControlCellKind::InhibitoryBasketSurround("iv", 3), 0)));
    lm.layer(LayerScheme::define("iii").depth(3).tags(LayerTags::PTAL).axon_domain(AxonDomain::output({THAL_SP}))
                 .cellular(CellScheme::pyramidal()
                     .tft(TuftScheme::basal().proximal().dens_per_tft(2).syns_per_den(16).thresh_init(8)
                         .src_lyr(TuftSourceLayer::define("iv").syn_reach(3).prevalence(1)))
                     .tft(TuftScheme::basal().distal().dens_per_tft(8).syns_per_den(16).max_active_dens_l2(2)
                         .thresh_init(4).src_lyr(TuftSourceLayer::define("iii").syn_reach(4).prevalence(1)))
                     .tft(TuftScheme::apical().distal().dens_per_tft(4).syns_per_den(12).max_active_dens_l2(1)
                         .src_lyr(TuftSourceLayer::define("ns_in").syn_reach(0).prevalence(1)))));
    lm.layer(LayerScheme::define("iii_out").cellular(CellScheme::control(ControlCellKind::PyrOutputter("iii"), 0)));
    lm.layer(LayerScheme::define("iii_col").cellular(CellScheme::control(ControlCellKind::IntraColumnInhib("iii"), 1)));
    lmaps.lmap(lm);
    areas.area(AreaScheme("v1", "visual", side).eff_areas({"v0"}));
}

LayerMapScheme hierarchy_map(const std::string& name, int depth, bool feedback) {
    LayerMapScheme lm(name, LayerMapKind::Cortical);
    lm.layer(LayerScheme::define("aff_in").axonal(AxonTopology::Spatial)
                 .axon_domain(AxonDomain::input({{InputTrack::Afferent, {THAL_SP}}})));
    if (feedback)
        lm.layer(LayerScheme::define("eff_in").axonal(AxonTopology::Spatial)
                     .axon_domain(AxonDomain::input({{InputTrack::Efferent, {THAL_SP}}})));
    lm.layer(LayerScheme::define("iv").depth(1).tags(LayerTags::PSAL).axon_domain(AxonDomain::Local())
                 .cellular(CellScheme::spiny_stellate().tft(TuftScheme::basal().proximal().syns_per_den(32)
                     .src_lyr(TuftSourceLayer::define("aff_in").syn_reach(6).prevalence(1)))));
    lm.layer(LayerScheme::define("iv_inhib")
                 .cellular(CellScheme::control(ControlCellKind::InhibitoryBasketSurround("iv", 4), 0)));
    CellScheme pyr = CellScheme::pyramidal()
        .tft(TuftScheme::basal().proximal().dens_per_tft(1).syns_per_den(1)
            .src_lyr(TuftSourceLayer::define("iv").syn_reach(0).prevalence(1)))
        .tft(TuftScheme::basal().distal().dens_per_tft(16).syns_per_den(32).max_active_dens_l2(3)
            .src_lyr(TuftSourceLayer::define("iii").syn_reach(6).prevalence(1)));
    if (feedback)
        pyr = pyr.tft(TuftScheme::apical().distal().dens_per_tft(16).syns_per_den(32).max_active_dens_l2(3)
                          .src_lyr(TuftSourceLayer::define("eff_in").syn_reach(6).prevalence(1)));
    lm.layer(LayerScheme::define("iii").depth(depth).tags(LayerTags::PTAL)
                 .axon_domain(AxonDomain::output({THAL_SP})).cellular(pyr));
    lm.layer(LayerScheme::define("iii_col")
                 .cellular(CellScheme::control(ControlCellKind::IntraColumnInhib("iii"), 0)));
    return lm;
}

// The three-area hierarchy (the Python configs.hierarchy).
std::vector<std::string> hierarchy(LayerMapSchemeList& lmaps, AreaSchemeList& areas,
                                   const std::vector<uint32_t>& sides, int depth) {
    external(lmaps, areas, "v0", sides[0]);
    lmaps.lmap(hierarchy_map("visual", depth, true));
    lmaps.lmap(hierarchy_map("visual_top", depth, false));
    std::vector<std::string> names;
    for (size_t k = 0; k < sides.size(); k++) names.push_back("v" + std::to_string(k + 1));
    for (size_t k = 0; k < sides.size(); k++) {
        const bool top = k + 1 == sides.size();
        AreaScheme a = AreaScheme(names[k], top ? "visual_top" : "visual", sides[k])
                           .eff_areas({k == 0 ? std::string("v0") : names[k - 1]});
        if (!top) a = a.aff_areas({names[k + 1]});
        areas.area(a);
    }
    return names;
}

CorticalAreaSettings settings() { return CorticalAreaSettings().disable_regrowth().strengths_start_at_zero(); }

void write_file(const std::string& path, const void* p, size_t n) {
    std::ofstream f(path, std::ios::binary);
    f.write((const char*)p, (std::streamsize)n);
}

std::vector<uint8_t> read_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    return std::vector<uint8_t>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

template <class F>
bool raises(int code, F&& f) {
    try {
        f();
    } catch (const CmnError& e) {
        return e.code == code;
    }
    return false;
}

int cmd_desc(const std::string& dir) {
    {
        LayerMapSchemeList lm;
        AreaSchemeList ar;
        benchmark_area(lm, ar, 64, 32, 1, 1, 1, 0);
        bm_area_desc d = area_desc("v1", lm, ar, settings());
        write_file(dir + "/area_64_v1.bin", &d, sizeof d);
    }
    {
        LayerMapSchemeList lm;
        AreaSchemeList ar;
        mixed_area(lm, ar, 32, 48);
        bm_area_desc d = area_desc("v1", lm, ar, settings());
        write_file(dir + "/mixed_v1.bin", &d, sizeof d);
    }
    {
        LayerMapSchemeList lm;
        AreaSchemeList ar;
        for (const auto& n : hierarchy(lm, ar, {32, 48, 24}, 2)) {
            bm_area_desc d = area_desc(n, lm, ar, settings());
            write_file(dir + "/hierarchy_" + n + ".bin", &d, sizeof d);
        }
    }
    {
        // The hierarchy with retina chains on an external, a feed-forward and
        // a feedback input.
        LayerMapSchemeList lm;
        AreaSchemeList ar;
        hierarchy(lm, ar, {32, 48, 24}, 2);
        AreaSchemeList ar2;
        for (const AreaScheme& a : ar.areas) {
            AreaScheme b = a;
            if (a.name == "v1") b = b.filter_chain(InputTrack::Afferent, {THAL_SP}, {FilterScheme("retina")});
            if (a.name == "v2")
                b = b.filter_chain(InputTrack::Afferent, {THAL_SP}, {FilterScheme("retina"), FilterScheme("retina")})
                        .filter_chain(InputTrack::Efferent, {THAL_SP}, {FilterScheme("retina")});
            ar2.area(b);
        }
        for (const char* n : {"v1", "v2"}) {
            bm_area_desc d = area_desc(n, lm, ar2, settings());
            write_file(dir + "/filtered_" + n + ".bin", &d, sizeof d);
        }
    }
    // Error behaviour: builder misuse and unresolvable schemes raise CmnError
    // with the C status code.
    bool ok = true;
    ok &= raises(BM_ERR_INVALID, [] { TuftSourceLayer::define("x").syn_reach(3).build(); });
    ok &= raises(BM_ERR_INVALID, [] { CellScheme::pyramidal().tft(TuftScheme::basal().syns_per_den(8)); });
    ok &= raises(BM_ERR_INVALID, [] { FilterScheme("sharpen"); });
    ok &= raises(BM_ERR_INVALID, [] { FilterScheme("retina", "my_filters.cl"); });
    ok &= raises(BM_ERR_INVALID, [] {
        LayerMapSchemeList lm;
        AreaSchemeList ar;
        benchmark_area(lm, ar, 64, 32, 1, 1, 1, 0);
        area_desc("v9", lm, ar, settings());
    });
    {
        // Regrowth on (the settings' default): the plan carries one
        // den_src_key0 byte per dendrite in every data layer.
        LayerMapSchemeList lm;
        AreaSchemeList ar;
        benchmark_area(lm, ar, 64, 32, 1, 1, 1, 0);
        bm_area_desc d = area_desc("v1", lm, ar, CorticalAreaSettings());
        bm_area_plan p;
        check(bm_plan_resolve(&d, 0, &p));
        for (uint32_t l = 0; l < p.n_layers; l++) ok &= p.layers[l].buf_len[BM_BUF_DEN_SRC_KEY0] == p.layers[l].n_dens;
    }
    std::cout << (ok ? "errors ok" : "errors WRONG") << std::endl;
    return ok ? 0 : 1;
}

int cmd_cycle(const std::string& dir) {
    LayerMapSchemeList lm;
    AreaSchemeList ar;
    auto names = hierarchy(lm, ar, {32, 48, 24}, 2);
    auto cx = Cortex::builder(lm, ar).ca_settings(settings()).seed(3).build();
    for (const auto& n : names) {
        auto s = cx->area(n).read_slab();
        write_file(dir + "/init_" + n + ".bin", s.data(), s.size());
    }
    if (cx->external_inputs().size() != 1 || cx->tracts().size() != 4) {
        std::cout << "routing WRONG" << std::endl;
        return 1;
    }
    const auto frames = read_file(dir + "/frames.bin");
    const size_t len = cx->external_inputs()[0].length;
    const size_t n = frames.size() / len;
    // A sampler on v2's axons: after each cycle it holds exactly what a read
    // of the same range returns.
    auto& v2 = cx->area("v2");
    Sampler& smp = v2.sampler(SamplerKind::Axons, BM_ALL_LAYERS);
    bool sampled = true;
    std::vector<uint8_t> frame;
    for (size_t c = 0; c < n; c++) {
        cx->area("v1").write_input(std::vector<uint8_t>(frames.begin() + c * len, frames.begin() + (c + 1) * len));
        cx->cycle();
        uint64_t cyc = 0;
        sampled = sampled && smp.recv(false, frame, &cyc) && cyc == c &&
                  frame == v2.read(BM_BUF_AXON_STATES, 0, 0, v2.plan().n_axons);
    }
    std::cout << (sampled ? "sampler ok" : "sampler WRONG") << std::endl;
    if (!sampled) return 1;
    for (const auto& a : names) {
        auto s = cx->area(a).read_slab();
        write_file(dir + "/final_" + a + ".bin", s.data(), s.size());
    }
    std::cout << "cycled " << n << std::endl;
    return cx->area("v1").cycle_count() == n ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::cerr << "usage: test_cortex desc|cycle <dir>" << std::endl;
        return 2;
    }
    try {
        const std::string cmd = argv[1];
        if (cmd == "desc") return cmd_desc(argv[2]);
        if (cmd == "cycle") return cmd_cycle(argv[2]);
    } catch (const CmnError& e) {
        std::cerr << "CmnError " << e.code << ": " << e.what() << std::endl;
        return 3;
    }
    return 2;
}
