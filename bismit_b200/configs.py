"""Area schemes for the benchmark workloads and the parity cases, plus seeded
synthetic input frames.

The benchmark area (one cortical area fed by a subcortical "external" area):

    aff_in   spatial input, depth 1, from the external area's THAL_SP output
    iv       spiny stellate (PSAL), depth 1, one basal proximal tuft
             1 x S synapses from aff_in, reach 6, threshold 0 (the default)
    iv_inhib InhibitoryBasketSurround on iv, radius 4
    iii      pyramidal (PTAL), depth D, output layer:
               basal proximal tuft from iv, basal distal tuft 16 x 32 from iii,
               reach 6, max_active_dens_l2 = 3
    iii_col  IntraColumnInhib on iii

Workload sizes:
  area_64   64 x 64 columns, S = 32, D = 1, proximal 1 x 1 reach 0
            (2,232,320 synapses)
  area_256  256 x 256 columns, S = 64, D = 4, proximal 16 x 32 reach 6
            (272,629,760 synapses)
Settings: regrowth disabled, learning on, strengths start at 0.
"""
import numpy as np

from .map import (AreaScheme, AreaSchemeList, AxonDomain, AxonTopology, CellScheme, ControlCellKind,
                  CorticalAreaSettings, InputTrack, LayerMapKind, LayerMapScheme, LayerMapSchemeList,
                  LayerScheme, LayerTags, THAL_NSP, THAL_SP, TuftScheme, TuftSourceLayer)


def _external(lmaps, areas, name, side, u_side=None, nonspatial=False, depth=1):
    lm = LayerMapScheme(name + "_lm", LayerMapKind.Subcortical)
    lm.layer(LayerScheme.define("ganglion").depth(depth).axonal(AxonTopology.Spatial)
             .axon_domain(AxonDomain.output([THAL_SP])))
    if nonspatial:
        lm.layer(LayerScheme.define("ganglion_ns").depth(1).axonal(AxonTopology.Nonspatial)
                 .axon_domain(AxonDomain.output([THAL_NSP])))
    lmaps.add(lm)
    areas.area(AreaScheme(name, lm.name, side, u_side))


def benchmark_area(side, ssc_syns, pyr_depth, prox_dens, prox_syns, prox_reach, name="v1"):
    """The benchmark layer map on a `side` x `side` area."""
    lmaps = LayerMapSchemeList()
    areas = AreaSchemeList()
    _external(lmaps, areas, "v0", side)
    lm = LayerMapScheme("visual", LayerMapKind.Cortical)
    lm.layer(LayerScheme.define("aff_in").axonal(AxonTopology.Spatial)
             .axon_domain(AxonDomain.input([(InputTrack.Afferent, [THAL_SP])])))
    lm.layer(LayerScheme.define("iv").depth(1).tags(LayerTags.PSAL).axon_domain(AxonDomain.Local)
             .cellular(CellScheme.spiny_stellate()
                       .tft(TuftScheme.basal().proximal().syns_per_den(ssc_syns)
                            .src_lyr(TuftSourceLayer.define("aff_in").syn_reach(6).prevalence(1)))))
    lm.layer(LayerScheme.define("iv_inhib")
             .cellular(CellScheme.control(ControlCellKind.InhibitoryBasketSurround("iv", 4), 0)))
    lm.layer(LayerScheme.define("iii").depth(pyr_depth).tags(LayerTags.PTAL)
             .axon_domain(AxonDomain.output([THAL_SP]))
             .cellular(CellScheme.pyramidal()
                       .tft(TuftScheme.basal().proximal().dens_per_tft(prox_dens).syns_per_den(prox_syns)
                            .src_lyr(TuftSourceLayer.define("iv").syn_reach(prox_reach).prevalence(1)))
                       .tft(TuftScheme.basal().distal().dens_per_tft(16).syns_per_den(32)
                            .max_active_dens_l2(3)
                            .src_lyr(TuftSourceLayer.define("iii").syn_reach(6).prevalence(1)))))
    lm.layer(LayerScheme.define("iii_col")
             .cellular(CellScheme.control(ControlCellKind.IntraColumnInhib("iii"), 0)))
    lmaps.add(lm)
    areas.area(AreaScheme(name, "visual", side).eff_areas(["v0"]))
    return lmaps, areas


def instance_area(side, depth, dens, syns, name="v1"):
    """One instance of the batched workload: the benchmark layer map with the
    64 x 64 area's shapes (spiny stellate 1 x 32, proximal 1 x 1 reach 0) on a
    `side` x `side` grid, pyramidal depth `depth` and a distal tuft of
    `dens` x `syns` (reach 6, max_active_dens_l2 = 3)."""
    lmaps = LayerMapSchemeList()
    areas = AreaSchemeList()
    _external(lmaps, areas, "v0", side)
    lm = LayerMapScheme("visual", LayerMapKind.Cortical)
    lm.layer(LayerScheme.define("aff_in").axonal(AxonTopology.Spatial)
             .axon_domain(AxonDomain.input([(InputTrack.Afferent, [THAL_SP])])))
    lm.layer(LayerScheme.define("iv").depth(1).tags(LayerTags.PSAL).axon_domain(AxonDomain.Local)
             .cellular(CellScheme.spiny_stellate()
                       .tft(TuftScheme.basal().proximal().syns_per_den(32)
                            .src_lyr(TuftSourceLayer.define("aff_in").syn_reach(6).prevalence(1)))))
    lm.layer(LayerScheme.define("iv_inhib")
             .cellular(CellScheme.control(ControlCellKind.InhibitoryBasketSurround("iv", 4), 0)))
    lm.layer(LayerScheme.define("iii").depth(depth).tags(LayerTags.PTAL)
             .axon_domain(AxonDomain.output([THAL_SP]))
             .cellular(CellScheme.pyramidal()
                       .tft(TuftScheme.basal().proximal().dens_per_tft(1).syns_per_den(1)
                            .src_lyr(TuftSourceLayer.define("iv").syn_reach(0).prevalence(1)))
                       .tft(TuftScheme.basal().distal().dens_per_tft(dens).syns_per_den(syns)
                            .max_active_dens_l2(3)
                            .src_lyr(TuftSourceLayer.define("iii").syn_reach(6).prevalence(1)))))
    lm.layer(LayerScheme.define("iii_col")
             .cellular(CellScheme.control(ControlCellKind.IntraColumnInhib("iii"), 0)))
    lmaps.add(lm)
    areas.area(AreaScheme(name, "visual", side).eff_areas(["v0"]))
    return lmaps, areas


def batch_instances(n=64, seed=0, sides=range(32, 193, 16)):
    """The batched workload: n independent instances, each drawn from a
    stream seeded by (seed, index): side uniform over `sides`, pyramidal depth
    1..4, distal dendrites per tuft from {8, 16}, synapses per dendrite from
    {16, 32, 64}, input activity uniform in [0.01, 0.04].
    Returns [(side, depth, dens, syns, active)]."""
    sides = list(sides)
    out = []
    for i in range(n):
        rng = np.random.default_rng([int(seed) & 0xFFFFFFFF, 0x62617463, i])
        out.append((int(sides[rng.integers(len(sides))]), int(rng.integers(1, 5)), int((8, 16)[rng.integers(2)]),
                    int((16, 32, 64)[rng.integers(3)]), float(rng.uniform(0.01, 0.04))))
    return out


def _hierarchy_map(name, depth, feedback):
    lm = LayerMapScheme(name, LayerMapKind.Cortical)
    lm.layer(LayerScheme.define("aff_in").axonal(AxonTopology.Spatial)
             .axon_domain(AxonDomain.input([(InputTrack.Afferent, [THAL_SP])])))
    if feedback:
        lm.layer(LayerScheme.define("eff_in").axonal(AxonTopology.Spatial)
                 .axon_domain(AxonDomain.input([(InputTrack.Efferent, [THAL_SP])])))
    lm.layer(LayerScheme.define("iv").depth(1).tags(LayerTags.PSAL).axon_domain(AxonDomain.Local)
             .cellular(CellScheme.spiny_stellate()
                       .tft(TuftScheme.basal().proximal().syns_per_den(32)
                            .src_lyr(TuftSourceLayer.define("aff_in").syn_reach(6).prevalence(1)))))
    lm.layer(LayerScheme.define("iv_inhib")
             .cellular(CellScheme.control(ControlCellKind.InhibitoryBasketSurround("iv", 4), 0)))
    pyr = (CellScheme.pyramidal()
           .tft(TuftScheme.basal().proximal().dens_per_tft(1).syns_per_den(1)
                .src_lyr(TuftSourceLayer.define("iv").syn_reach(0).prevalence(1)))
           .tft(TuftScheme.basal().distal().dens_per_tft(16).syns_per_den(32).max_active_dens_l2(3)
                .src_lyr(TuftSourceLayer.define("iii").syn_reach(6).prevalence(1))))
    if feedback:
        pyr.tft(TuftScheme.apical().distal().dens_per_tft(16).syns_per_den(32).max_active_dens_l2(3)
                .src_lyr(TuftSourceLayer.define("eff_in").syn_reach(6).prevalence(1)))
    lm.layer(LayerScheme.define("iii").depth(depth).tags(LayerTags.PTAL)
             .axon_domain(AxonDomain.output([THAL_SP])).cellular(pyr))
    lm.layer(LayerScheme.define("iii_col")
             .cellular(CellScheme.control(ControlCellKind.IntraColumnInhib("iii"), 0)))
    return lm


def hierarchy(sides=(128, 192, 96), depth=2):
    """The three-area hierarchy: cortical areas v1 -> v2 -> v3 of the given
    sides, fed by an external area v0 the size of v1. Each area has the 64 x 64
    area's layer shapes at pyramidal depth `depth`; its feed-forward input
    `aff_in` comes from the previous area's output layer iii. Every area but
    the top one also has an efferent input `eff_in`, fed back from the next
    area's iii, which an apical distal tuft (16 x 32, reach 6) samples: bismit
    requires the source slices of one tuft to offer equal offset pools
    (SynSrcSlices::new), which slices of another area's scale do not, so the
    feedback gets a tuft of its own. Returns (lmaps, areas, cortical area
    names in order)."""
    lmaps = LayerMapSchemeList()
    areas = AreaSchemeList()
    _external(lmaps, areas, "v0", sides[0])
    lmaps.add(_hierarchy_map("visual", depth, True))
    lmaps.add(_hierarchy_map("visual_top", depth, False))
    names = ["v%d" % (k + 1) for k in range(len(sides))]
    for k, (n, side) in enumerate(zip(names, sides)):
        top = k + 1 == len(names)
        a = AreaScheme(n, "visual_top" if top else "visual", side).eff_areas(["v0" if k == 0 else names[k - 1]])
        if not top:
            a.aff_areas([names[k + 1]])
        areas.area(a)
    return lmaps, areas, names


def bench_settings():
    return CorticalAreaSettings().disable_regrowth().strengths_start_at_zero()


WORKLOADS = {
    # name: (side, ssc_syns, pyr_depth, prox_dens, prox_syns, prox_reach, input active fraction)
    "area_64": (64, 32, 1, 1, 1, 0, 0.02),
    "area_256": (256, 64, 4, 16, 32, 6, 0.03),
    "area_128": (128, 32, 2, 1, 1, 0, 0.02),
    "area_32": (32, 32, 1, 1, 1, 0, 0.02),
    "area_48_deep": (48, 32, 2, 4, 16, 3, 0.03),
    "area_256_shape": (48, 64, 4, 16, 32, 6, 0.03),
}


def workload(name):
    side, s, d, pd, ps, pr, act = WORKLOADS[name]
    lmaps, areas = benchmark_area(side, s, d, pd, ps, pr)
    return lmaps, areas, act


def testbed_area(side=24, retina=False):
    """The reference's test bed layer map (src/tests/testbed.rs:18-208):
    spatial input, a spiny stellate layer with a threshold of 400, basket
    inhibition and a 3-deep pyramidal layer with a basal distal and an apical
    distal tuft (both learn, in tuft order); with `retina`, also its retina
    filter chain on the afferent input (testbed.rs:188)."""
    lmaps = LayerMapSchemeList()
    areas = AreaSchemeList()
    _external(lmaps, areas, "v0", side)
    lm = LayerMapScheme("visual", LayerMapKind.Cortical)
    lm.layer(LayerScheme.define("motor_in").depth(1).axonal(AxonTopology.Nonspatial)
             .axon_domain(AxonDomain.input([(InputTrack.Afferent, ["thal_motor"])])))
    lm.layer(LayerScheme.define("eff_in").axonal(AxonTopology.Spatial)
             .axon_domain(AxonDomain.input([(InputTrack.Efferent, [THAL_SP])])))
    lm.layer(LayerScheme.define("aff_in").axonal(AxonTopology.Spatial)
             .axon_domain(AxonDomain.input([(InputTrack.Afferent, [THAL_SP])])))
    lm.layer(LayerScheme.define("out").depth(1).axonal(AxonTopology.Spatial)
             .axon_domain(AxonDomain.output([THAL_SP])))
    lm.layer(LayerScheme.define("unused").depth(1).tags(LayerTags.UNUSED).axonal(AxonTopology.Spatial)
             .axon_domain(AxonDomain.Local))
    lm.layer(LayerScheme.define("iv").depth(1).tags(LayerTags.PSAL).axon_domain(AxonDomain.Local)
             .cellular(CellScheme.spiny_stellate()
                       .tft(TuftScheme.basal().proximal().syns_per_den(32).thresh_init(400)
                            .src_lyr(TuftSourceLayer.define("aff_in").syn_reach(8).prevalence(1)))))
    lm.layer(LayerScheme.define("iv_inhib")
             .cellular(CellScheme.control(ControlCellKind.InhibitoryBasketSurround("iv", 4), 0)))
    lm.layer(LayerScheme.define("iii").depth(3).tags(LayerTags.PTAL).axon_domain(AxonDomain.Local)
             .cellular(CellScheme.pyramidal()
                       .tft(TuftScheme.basal().distal().dens_per_tft(4).syns_per_den(8).max_active_dens_l2(0)
                            .thresh_init(1200).src_lyr(TuftSourceLayer.define("iii").syn_reach(16).prevalence(1)))
                       .tft(TuftScheme.apical().distal().dens_per_tft(2).syns_per_den(32).max_active_dens_l2(0)
                            .thresh_init(500).src_lyr(TuftSourceLayer.define("iii").syn_reach(3).prevalence(1)))))
    lmaps.add(lm)
    a = AreaScheme("v1", "visual", side).eff_areas(["v0"])
    if retina:
        a.filter_chain(InputTrack.Afferent, [THAL_SP], [("retina", None)])
    areas.area(a)
    return lmaps, areas


def retina_area(side=48, n_filters=1, src_depth=1, src_side=None):
    """An instance-style area whose afferent input passes through a chain of
    `n_filters` retina filters (cl/filters.cl:34-100) from a source `src_depth`
    slices deep and `src_side` wide (default: the area's side)."""
    lmaps = LayerMapSchemeList()
    areas = AreaSchemeList()
    _external(lmaps, areas, "v0", src_side or side, depth=src_depth)
    lm = LayerMapScheme("visual", LayerMapKind.Cortical)
    lm.layer(LayerScheme.define("aff_in").axonal(AxonTopology.Spatial)
             .axon_domain(AxonDomain.input([(InputTrack.Afferent, [THAL_SP])])))
    lm.layer(LayerScheme.define("iv").depth(1).tags(LayerTags.PSAL).axon_domain(AxonDomain.Local)
             .cellular(CellScheme.spiny_stellate()
                       .tft(TuftScheme.basal().proximal().syns_per_den(32)
                            .src_lyr(TuftSourceLayer.define("aff_in").syn_reach(6).prevalence(1)))))
    lm.layer(LayerScheme.define("iv_inhib")
             .cellular(CellScheme.control(ControlCellKind.InhibitoryBasketSurround("iv", 4), 0)))
    lm.layer(LayerScheme.define("iii").depth(2).tags(LayerTags.PTAL).axon_domain(AxonDomain.output([THAL_SP]))
             .cellular(CellScheme.pyramidal()
                       .tft(TuftScheme.basal().proximal().dens_per_tft(1).syns_per_den(1)
                            .src_lyr(TuftSourceLayer.define("iv").syn_reach(0).prevalence(1)))
                       .tft(TuftScheme.basal().distal().dens_per_tft(8).syns_per_den(32).max_active_dens_l2(3)
                            .src_lyr(TuftSourceLayer.define("iii").syn_reach(6).prevalence(1)))))
    lm.layer(LayerScheme.define("iii_col")
             .cellular(CellScheme.control(ControlCellKind.IntraColumnInhib("iii"), 0)))
    lmaps.add(lm)
    areas.area(AreaScheme("v1", "visual", side).eff_areas(["v0"])
               .filter_chain(InputTrack.Afferent, [THAL_SP], ["retina"] * n_filters))
    return lmaps, areas


def smoother_area(side=40, radius=3, pyr_radius=2, smoothers=True):
    """An instance-style layer map with ActivitySmoother control layers
    (src/cortex/smoother.rs): one on the spiny stellate layer after its basket
    inhibition, one on the pyramidal layer after its intra-column inhibition.
    Group side `radius` / `pyr_radius`."""
    lmaps = LayerMapSchemeList()
    areas = AreaSchemeList()
    _external(lmaps, areas, "v0", side)
    lm = LayerMapScheme("visual", LayerMapKind.Cortical)
    lm.layer(LayerScheme.define("aff_in").axonal(AxonTopology.Spatial)
             .axon_domain(AxonDomain.input([(InputTrack.Afferent, [THAL_SP])])))
    lm.layer(LayerScheme.define("iv").depth(1).tags(LayerTags.PSAL).axon_domain(AxonDomain.Local)
             .cellular(CellScheme.spiny_stellate()
                       .tft(TuftScheme.basal().proximal().syns_per_den(32)
                            .src_lyr(TuftSourceLayer.define("aff_in").syn_reach(6).prevalence(1)))))
    lm.layer(LayerScheme.define("iv_inhib")
             .cellular(CellScheme.control(ControlCellKind.InhibitoryBasketSurround("iv", 4), 0)))
    lm.layer(LayerScheme.define("iii").depth(2).tags(LayerTags.PTAL).axon_domain(AxonDomain.output([THAL_SP]))
             .cellular(CellScheme.pyramidal()
                       .tft(TuftScheme.basal().proximal().dens_per_tft(1).syns_per_den(1)
                            .src_lyr(TuftSourceLayer.define("iv").syn_reach(0).prevalence(1)))
                       .tft(TuftScheme.basal().distal().dens_per_tft(8).syns_per_den(32).max_active_dens_l2(3)
                            .src_lyr(TuftSourceLayer.define("iii").syn_reach(6).prevalence(1)))))
    lm.layer(LayerScheme.define("iii_col")
             .cellular(CellScheme.control(ControlCellKind.IntraColumnInhib("iii"), 0)))
    if smoothers:   # last, so that every other layer keeps its id (and its random streams)
        lm.layer(LayerScheme.define("iv_smooth")
                 .cellular(CellScheme.control(ControlCellKind.ActivitySmoother("iv", radius), 1)))
        lm.layer(LayerScheme.define("iii_smooth")
                 .cellular(CellScheme.control(ControlCellKind.ActivitySmoother("iii", pyr_radius), 1)))
    lmaps.add(lm)
    areas.area(AreaScheme("v1", "visual", side).eff_areas(["v0"]))
    return lmaps, areas


def mixed_area(side=32, src_side=48):
    """A parity case that exercises the remaining index and control paths:
    a scaled input slice (source area larger than the area), a nonspatial input
    slice, prevalence repeats, a proximal+distal+apical pyramidal layer whose
    two distal tufts learn in order, PyrOutputter followed by IntraColumnInhib
    on the same host, and non-zero dendrite thresholds."""
    lmaps = LayerMapSchemeList()
    areas = AreaSchemeList()
    _external(lmaps, areas, "v0", src_side, nonspatial=True)
    lm = LayerMapScheme("visual", LayerMapKind.Cortical)
    lm.layer(LayerScheme.define("aff_in").axonal(AxonTopology.Spatial)
             .axon_domain(AxonDomain.input([(InputTrack.Afferent, [THAL_SP])])))
    lm.layer(LayerScheme.define("ns_in").axonal(AxonTopology.Nonspatial)
             .axon_domain(AxonDomain.input([(InputTrack.Afferent, [THAL_NSP])])))
    lm.layer(LayerScheme.define("iv").depth(2).tags(LayerTags.PSAL)
             .cellular(CellScheme.spiny_stellate()
                       .tft(TuftScheme.basal().proximal().syns_per_den(24).thresh_init(40)
                            .src_lyr(TuftSourceLayer.define("aff_in").syn_reach(4).prevalence(2)))))
    lm.layer(LayerScheme.define("iv_inhib")
             .cellular(CellScheme.control(ControlCellKind.InhibitoryBasketSurround("iv", 3), 0)))
    lm.layer(LayerScheme.define("iii").depth(3).tags(LayerTags.PTAL).axon_domain(AxonDomain.output([THAL_SP]))
             .cellular(CellScheme.pyramidal()
                       .tft(TuftScheme.basal().proximal().dens_per_tft(2).syns_per_den(16).thresh_init(8)
                            .src_lyr(TuftSourceLayer.define("iv").syn_reach(3).prevalence(1)))
                       .tft(TuftScheme.basal().distal().dens_per_tft(8).syns_per_den(16).max_active_dens_l2(2)
                            .thresh_init(4).src_lyr(TuftSourceLayer.define("iii").syn_reach(4).prevalence(1)))
                       .tft(TuftScheme.apical().distal().dens_per_tft(4).syns_per_den(12).max_active_dens_l2(1)
                            .src_lyr(TuftSourceLayer.define("ns_in").syn_reach(0).prevalence(1)))))
    lm.layer(LayerScheme.define("iii_out")
             .cellular(CellScheme.control(ControlCellKind.PyrOutputter("iii"), 0)))
    lm.layer(LayerScheme.define("iii_col")
             .cellular(CellScheme.control(ControlCellKind.IntraColumnInhib("iii"), 1)))
    lmaps.add(lm)
    areas.area(AreaScheme("v1", "visual", side).eff_areas(["v0"]))
    return lmaps, areas


def frames(n, length, active, seed, start=0):
    """n seeded u8 frames: each axon active with probability `active`, active
    values uniform in 1..255 (frame k depends only on (seed, start + k))."""
    out = np.zeros((n, length), dtype=np.uint8)
    for k in range(n):
        rng = np.random.default_rng([int(seed) & 0xFFFFFFFF, 0x6672616D, start + k])
        m = rng.random(length) < active
        out[k, m] = rng.integers(1, 256, size=int(m.sum()), dtype=np.uint16).astype(np.uint8)
    return out
