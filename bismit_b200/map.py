"""Layer-map and area schemes: the builder API of bismit's `map` module.

Mirrors src/map/scheme/{layer_map,layer,cell,area}.rs (same builder names and
argument meanings) and resolves a cortical area into the C descriptor
(bm_area_desc) the native library takes. Input-layer sources are resolved the
way LayerInfo::new does (src/map/layer_info.rs:14-100,142-215): for each input
signature (track, axon tags) the candidate areas are the area's efferent areas
(afferent track) or afferent areas (efferent track), and every output layer of
those areas with matching axon tags contributes one slice range.
"""
import ctypes as C

from . import _ffi as F

# ------------------------------------------------------------------ tags ----


class LayerTags:
    """Bit flags of src/map/layer_tags.rs:121-150 (high word)."""
    DEFAULT = 0
    PRIMARY = F.BM_TAG_PRIMARY
    SPATIAL = F.BM_TAG_SPATIAL
    TEMPORAL = F.BM_TAG_TEMPORAL
    FOCUS = F.BM_TAG_FOCUS
    MOTOR = F.BM_TAG_MOTOR
    UNUSED = F.BM_TAG_UNUSED
    INPUT = F.BM_TAG_INPUT
    OUTPUT = F.BM_TAG_OUTPUT
    PSAL = F.BM_TAG_PRIMARY | F.BM_TAG_SPATIAL
    PTAL = F.BM_TAG_PRIMARY | F.BM_TAG_TEMPORAL
    PFL = F.BM_TAG_PRIMARY | F.BM_TAG_FOCUS
    PML = F.BM_TAG_PRIMARY | F.BM_TAG_MOTOR


# Axon tags (src/map/axon_tags.rs:55-57).
THAL_SP = "thal_sp"
THAL_NSP = "thal_nsp"
THAL_ASC = "thal_asc"


class AxonTopology:
    Spatial = F.BM_TOPO_SPATIAL
    Nonspatial = F.BM_TOPO_NONSPATIAL
    None_ = F.BM_TOPO_NONE


class InputTrack:
    Afferent = "afferent"
    Efferent = "efferent"
    Other = "other"


class AxonDomain:
    """AxonDomain::{Local, input(..), output(..)} (src/map/mod.rs)."""

    def __init__(self, kind, sigs=()):
        self.kind = kind
        self.sigs = list(sigs)

    @staticmethod
    def input(sigs):
        out = []
        for track, tags in sigs:
            out.append((track, frozenset(tags)))
        return AxonDomain(F.BM_DOM_INPUT, out)

    @staticmethod
    def output(tags):
        return AxonDomain(F.BM_DOM_OUTPUT, [(None, frozenset(tags))])


AxonDomain.Local = AxonDomain(F.BM_DOM_LOCAL)


class LayerMapKind:
    Cortical = "cortical"
    Subcortical = "subcortical"


# ----------------------------------------------------------- cell schemes --


class TuftSourceLayer:
    """TuftSourceLayer::define(name).syn_reach(r).prevalence(p) (src/map/scheme/cell.rs:6-92)."""

    def __init__(self, name):
        self.name = name
        self._reach = None
        self._prevalence = None

    @staticmethod
    def define(name):
        return TuftSourceLayer(name)

    def syn_reach(self, r):
        self._reach = int(r)
        return self

    def prevalence(self, p):
        self._prevalence = int(p)
        return self

    def build(self):
        if self._reach is None or self._prevalence is None:
            raise ValueError("TuftSourceLayerDefinition::build: syn_reach and prevalence are required")
        if self._prevalence < 1:
            raise ValueError("Tuft source layer definitions must have a prevalence of at least one.")
        return self


class TuftScheme:
    """TuftScheme builder (src/map/scheme/cell.rs:95-263)."""

    def __init__(self):
        self.den_class = None
        self.den_kind = None
        self._dens_per_tft = 1
        self._syns_per_den = None
        self._max_active_dens_l2 = 0
        self.src_lyrs = []
        self._thresh_init = None

    @staticmethod
    def basal():
        t = TuftScheme()
        t.den_class = F.BM_DEN_BASAL
        return t

    @staticmethod
    def apical():
        t = TuftScheme()
        t.den_class = F.BM_DEN_APICAL
        return t

    def proximal(self):
        self.den_kind = F.BM_DEN_PROXIMAL
        return self

    def distal(self):
        self.den_kind = F.BM_DEN_DISTAL
        return self

    def dens_per_tft(self, n):
        self._dens_per_tft = int(n)
        return self

    def syns_per_den(self, n):
        self._syns_per_den = int(n)
        return self

    def max_active_dens_l2(self, n):
        self._max_active_dens_l2 = int(n)
        return self

    def thresh_init(self, n):
        self._thresh_init = int(n)
        return self

    def src_lyr(self, src):
        self.src_lyrs.append(src.build())
        return self

    def syns_per_tft(self):
        return self._dens_per_tft * self._syns_per_den


class ControlCellKind:
    """ControlCellKind variants on this path (src/map/mod.rs)."""

    class InhibitoryBasketSurround:
        def __init__(self, host_lyr_name, field_radius):
            self.host_lyr_name = host_lyr_name
            self.field_radius = int(field_radius)
            self.kind = F.BM_LYR_CTRL_INHIB_BASKET

    class PyrOutputter:
        def __init__(self, host_lyr_name):
            self.host_lyr_name = host_lyr_name
            self.field_radius = 0
            self.kind = F.BM_LYR_CTRL_PYR_OUTPUT

    class IntraColumnInhib:
        def __init__(self, host_lyr_name):
            self.host_lyr_name = host_lyr_name
            self.field_radius = 0
            self.kind = F.BM_LYR_CTRL_INTRA_COLUMN

    class ActivitySmoother:
        def __init__(self, host_lyr_name, field_radius):
            self.host_lyr_name = host_lyr_name
            self.field_radius = int(field_radius)
            self.kind = F.BM_LYR_CTRL_SMOOTHER


class CellScheme:
    """CellScheme::{spiny_stellate, pyramidal, control} (src/map/scheme/cell.rs)."""

    def __init__(self, kind):
        self.kind = kind
        self.tfts = []
        self.control = None
        self.exe_order = 0

    @staticmethod
    def spiny_stellate():
        return CellScheme(F.BM_LYR_SPINY_STELLATE)

    @staticmethod
    def pyramidal():
        return CellScheme(F.BM_LYR_PYRAMIDAL)

    @staticmethod
    def control(kind, exe_order):
        c = CellScheme(kind.kind)
        c.control = kind
        c.exe_order = int(exe_order)
        return c

    def tft(self, tft_scheme):
        if tft_scheme.den_class is None or tft_scheme.den_kind is None or tft_scheme._syns_per_den is None:
            raise ValueError("TuftScheme::build: class, kind and syns_per_den are required")
        self.tfts.append(tft_scheme)
        return self


class LayerScheme:
    """LayerScheme::define(name)... (src/map/scheme/layer.rs:42-130)."""

    def __init__(self, name):
        self.name = name
        self._depth = None
        self._tags = LayerTags.DEFAULT
        self.kind = F.BM_LYR_AXONAL
        self.axon_topology = AxonTopology.Spatial
        self._axon_domain = AxonDomain.Local
        self.cell_scheme = None

    @staticmethod
    def define(name):
        return LayerScheme(name)

    def depth(self, d):
        self._depth = int(d)
        return self

    def tags(self, t):
        self._tags = int(t)
        return self

    def axonal(self, topology):
        self.kind = F.BM_LYR_AXONAL
        self.axon_topology = topology
        return self

    def axon_domain(self, dom):
        self._axon_domain = dom
        return self

    def cellular(self, cell_scheme):
        self.cell_scheme = cell_scheme
        self.kind = cell_scheme.kind
        return self


class LayerMapScheme:
    def __init__(self, name, kind=LayerMapKind.Cortical):
        self.name = name
        self.kind = kind
        self.layers = []

    def layer(self, ls):
        self.layers.append(ls)
        return self

    def output_layers_with_axon_tags(self, tags):
        out = []
        for ls in self.layers:
            d = ls._axon_domain
            if d.kind == F.BM_DOM_OUTPUT and any(tags <= t for _, t in d.sigs):
                out.append(ls)
        return out


class LayerMapSchemeList:
    def __init__(self):
        self.maps = {}

    def add(self, lms):
        self.maps[lms.name] = lms
        return self

    lmap = add

    def __getitem__(self, name):
        return self.maps[name]


class FilterScheme:
    """FilterScheme::new(filter_name, cl_file_name) (src/map/scheme/filter.rs:3-40):
    one filter of an input filter chain, named by its kernel. The built-in
    filter is "retina" (cl/filters.cl:34-100); a kernel from a custom OpenCL
    file has no counterpart here."""

    KINDS = {"retina": F.BM_FILTER_RETINA}

    def __init__(self, filter_name, cl_file_name=None):
        if filter_name not in self.KINDS:
            raise ValueError("unknown filter %r (built in: %s)" % (filter_name, ", ".join(sorted(self.KINDS))))
        if cl_file_name is not None:
            raise ValueError("filter %r: kernels from custom OpenCL files are not supported" % filter_name)
        self.filter_name = filter_name
        self.cl_file_name = cl_file_name

    @property
    def kind(self):
        return self.KINDS[self.filter_name]


class AreaScheme:
    """AreaScheme::new(name, layer_map_name, side) (src/map/scheme/area.rs:22-198)."""

    def __init__(self, name, layer_map_name, side, u_side=None):
        self.name = name
        self.layer_map_name = layer_map_name
        self.v_size = int(side)
        self.u_size = int(side if u_side is None else u_side)
        self._eff_areas = []
        self._aff_areas = []
        self._other_areas = []
        self._filter_chains = []

    def filter_chain(self, input_track, axn_tags, filter_chain):
        """AreaScheme::filter_chain (src/map/scheme/area.rs:70-85): frames of
        the source matched by the input signature (input_track, axn_tags) pass
        through the filters in order. Each filter is a FilterScheme, a
        (name, cl_file_name) pair or a name."""
        chain = []
        for f in filter_chain:
            if isinstance(f, FilterScheme):
                chain.append(f)
            elif isinstance(f, tuple):
                chain.append(FilterScheme(*f))
            else:
                chain.append(FilterScheme(f))
        if len(chain) > F.BM_MAX_FILTERS:
            raise ValueError("more than %d filters in one chain" % F.BM_MAX_FILTERS)
        self._filter_chains.append((input_track, frozenset(axn_tags), chain))
        return self

    @staticmethod
    def irregular(name, layer_map_name, dims):
        return AreaScheme(name, layer_map_name, dims[0], dims[1])

    def eff_areas(self, names):
        self._eff_areas = list(names)
        return self

    def aff_areas(self, names):
        self._aff_areas = list(names)
        return self

    def other_areas(self, names):
        self._other_areas = list(names)
        return self


class AreaSchemeList:
    def __init__(self):
        self.areas = []

    def area(self, a):
        self.areas.append(a)
        return self

    def by_name(self, name):
        for a in self.areas:
            if a.name == name:
                return a
        raise KeyError(name)

    def area_id(self, name):
        for i, a in enumerate(self.areas):
            if a.name == name:
                return i
        raise KeyError(name)


class CorticalAreaSettings:
    """CorticalAreaSettings (src/cortex/cortical_area.rs:253-338)."""

    def __init__(self):
        self.bits = 0
        self.init_flags = 0
        self.exec_path = F.BM_PATH_FUSED

    def _set(self, b):
        self.bits |= b
        return self

    def bypass_inhib(self):
        return self._set(F.BM_SET_BYPASS_INHIB)

    def bypass_filters(self):
        return self._set(F.BM_SET_BYPASS_FILTERS)

    def disable_pyrs(self):
        return self._set(F.BM_SET_DISABLE_PYRS)

    def disable_sscs(self):
        return self._set(F.BM_SET_DISABLE_SSCS)

    def disable_mcols(self):
        return self._set(F.BM_SET_DISABLE_MCOLS)

    def disable_regrowth(self):
        return self._set(F.BM_SET_DISABLE_REGROWTH)

    def disable_learning(self):
        return self._set(F.BM_SET_DISABLE_LEARNING)

    def strengths_start_at_zero(self):
        self.init_flags |= F.BM_INIT_STRENGTH_ZERO
        return self

    def plain_kernels(self):
        """Runs one kernel per reference stage instead of the fused kernels."""
        self.exec_path = F.BM_PATH_PLAIN
        return self


# -------------------------------------------------------------- resolution --

def source_list(area_sch, area_list, lmaps, sigs):
    """matching_source_layers, src/map/layer_info.rs:14-100: the source layers
    feeding an input layer with signatures `sigs`, in slice order, as
    (source area name, source layer name, v_size, u_size, depth, topology)."""
    out = []
    for track, tags in sigs:
        if track == InputTrack.Afferent:
            cands = area_sch._eff_areas
        elif track == InputTrack.Efferent:
            cands = area_sch._aff_areas
        else:
            cands = area_sch._other_areas
        for an in cands:
            src_area = area_list.by_name(an)
            src_map = lmaps[src_area.layer_map_name]
            for ls in src_map.output_layers_with_axon_tags(tags):
                depth = ls._depth if ls._depth is not None else 1   # DEFAULT_OUTPUT_LAYER_DEPTH
                topo = ls.axon_topology if ls.kind == F.BM_LYR_AXONAL else AxonTopology.Spatial
                out.append((an, ls.name, src_area.v_size, src_area.u_size, depth, topo))
    return out


def _source_layers(area_sch, area_list, lmaps, sigs):
    return [x[2:] for x in source_list(area_sch, area_list, lmaps, sigs)]


def _attach_filter_chains(d, a, areas, lmaps, lm):
    """Each filter chain of area scheme `a` goes to the one source whose input
    signature it names (AxonSpace::new, src/cortex/axon_space.rs:340-345, with
    LayerMap::src_layer_info_by_sig, src/map/layer_map.rs:242-261)."""
    for track, tags, chain in a._filter_chains:
        hits = []
        for i, ls in enumerate(lm.layers):
            if ls._axon_domain.kind != F.BM_DOM_INPUT:
                continue
            k = 0
            for sig in ls._axon_domain.sigs:
                n = len(source_list(a, areas, lmaps, [sig]))
                if sig == (track, tags):
                    hits += [(i, k + j) for j in range(n)]
                k += n
        if not hits:
            raise ValueError("Unable to find a layer within the area map matching the axon domain "
                             "(track: %r, tags: %r) specified by the filter chain scheme." % (track, sorted(tags)))
        if len(hits) > 1:
            raise ValueError("Duplicate axon signatures (%r, %r) found within the layer map for area %r."
                             % (track, sorted(tags), a.name))
        i, k = hits[0]
        S = d.layers[i].input_srcs[k]
        if S.n_filters:
            raise ValueError("two filter chains for the source (%r, %r)" % (track, sorted(tags)))
        S.n_filters = len(chain)
        for j, f in enumerate(chain):
            S.filters[j] = f.kind


def area_desc(area_name, lmaps, areas, settings=None, area_id=None):
    """Resolves one cortical area of `areas` into a bm_area_desc."""
    settings = settings or CorticalAreaSettings().disable_regrowth()
    a = areas.by_name(area_name)
    lm = lmaps[a.layer_map_name]
    if lm.kind != LayerMapKind.Cortical:
        raise ValueError("area %r has a subcortical layer map" % area_name)
    if len(lm.layers) > F.BM_MAX_LAYERS:
        raise ValueError("too many layers")
    d = F.bm_area_desc()
    d.area_id = areas.area_id(area_name) if area_id is None else area_id
    d.v_size, d.u_size = a.v_size, a.u_size
    d.n_layers = len(lm.layers)
    d.settings = settings.bits
    d.init_flags = settings.init_flags
    d.exec_path = settings.exec_path
    idx = {ls.name: i for i, ls in enumerate(lm.layers)}
    for i, ls in enumerate(lm.layers):
        L = d.layers[i]
        name = ls.name.encode()
        if len(name) >= F.BM_NAME_LEN:
            raise ValueError("layer name too long: %r" % ls.name)
        L.name = name
        L.tags = ls._tags
        L.kind = ls.kind
        L.depth = -1 if ls._depth is None else ls._depth
        L.axon_topology = ls.axon_topology
        L.axon_domain = ls._axon_domain.kind
        L.host_layer_idx = -1
        if ls._axon_domain.kind == F.BM_DOM_INPUT:
            srcs = _source_layers(a, areas, lmaps, ls._axon_domain.sigs)
            if len(srcs) > F.BM_MAX_IO:
                raise ValueError("too many input sources")
            L.n_input_srcs = len(srcs)
            for k, (v, u, dep, topo) in enumerate(srcs):
                L.input_srcs[k] = F.bm_input_src_desc(v, u, dep, topo)
        cs = ls.cell_scheme
        if cs is not None and cs.control is not None:
            L.host_layer_idx = idx[cs.control.host_lyr_name]
            L.field_radius = cs.control.field_radius
            L.exe_order = cs.exe_order
        elif cs is not None:
            if len(cs.tfts) > F.BM_MAX_TUFTS:
                raise ValueError("too many tufts")
            L.n_tufts = len(cs.tfts)
            for t, ts in enumerate(cs.tfts):
                T = L.tufts[t]
                T.den_class, T.den_kind = ts.den_class, ts.den_kind
                T.dens_per_tft, T.syns_per_den = ts._dens_per_tft, ts._syns_per_den
                T.max_active_dens_l2 = ts._max_active_dens_l2
                T.thresh_init = -1 if ts._thresh_init is None else ts._thresh_init
                if len(ts.src_lyrs) > F.BM_MAX_SRC_LAYERS:
                    raise ValueError("too many tuft sources")
                T.n_src = len(ts.src_lyrs)
                for k, sl in enumerate(ts.src_lyrs):
                    if sl.name not in idx:
                        raise ValueError("tuft source layer %r not in the layer map" % sl.name)
                    T.src[k] = F.bm_src_layer_desc(idx[sl.name], sl._reach, sl._prevalence)
    _attach_filter_chains(d, a, areas, lmaps, lm)
    return d


def area_tracts(lmaps, areas, names, plans):
    """Thalamic routing among the cortical areas `names` (plans[k] resolves
    names[k]): every input layer's source slices in order (LayerInfo::new,
    src/map/layer_info.rs:142-215), each either a tract from another area of
    `names` or an external feed. Returns (tracts, external) with
    tracts = [(src_k, src_output, dst_k, dst_input, dst_offset, length)] and
    external = [(dst_k, dst_input, dst_offset, length, source area, source layer)]."""
    tracts, external = [], []
    pos = {n: k for k, n in enumerate(names)}
    for k, n in enumerate(names):
        a = areas.by_name(n)
        lm = lmaps[a.layer_map_name]
        P = plans[k]
        for i in range(P.n_inputs):
            ls = lm.layers[P.inputs[i].layer_idx]
            off = 0
            for (src, src_layer, v, u, dep, _topo) in source_list(a, areas, lmaps, ls._axon_domain.sigs):
                length = v * u * dep
                if src in pos:
                    S = plans[pos[src]]
                    src_lm = lmaps[areas.by_name(src).layer_map_name]
                    li = [x.name for x in src_lm.layers].index(src_layer)
                    o = [S.outputs[j].layer_idx for j in range(S.n_outputs)].index(li)
                    if int(S.outputs[o].len) != length:
                        raise ValueError("tract %s.%s -> %s: %d axons, expected %d" % (src, src_layer, n,
                                                                                     S.outputs[o].len, length))
                    tracts.append((pos[src], o, k, i, off, length))
                else:
                    external.append((k, i, off, length, src, src_layer))
                off += length
            if off != int(P.inputs[i].len):
                raise ValueError("input %d of %s: sources give %d axons, plan has %d" % (i, n, off, P.inputs[i].len))
    return tracts, external


def desc_layer_index(desc, name):
    for i in range(desc.n_layers):
        if desc.layers[i].name.decode() == name:
            return i
    raise KeyError(name)
