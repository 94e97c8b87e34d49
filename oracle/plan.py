"""The oracle's own plan resolver (TEST INFRASTRUCTURE): an area scheme
(bm_area_desc) to the plan of slice tables, index spaces and state-slab
offsets (bm_area_plan), restated in Python from bismit's host-side map code so
that the oracle and the CPU reference arm need nothing from the library:

  LayerMap::new, LayerInfo::new      src/map/layer_map.rs:66-100, src/map/layer_info.rs:116-300
  SliceMap::new                      src/map/slice_map.rs:26-156
  SliceDims::new, calc_scale         src/cmn/slice_dims.rs:20-121, :201-224
  AreaMap::cel_src_slc_id_rchs       src/map/area_map.rs:139-162
  SynSrcSlices::new, gen_syn_offs    src/map/syn_src.rs:390-446, :47-149
  Synapses / Dendrites / Tufts index spaces
                                     src/cortex/synapses.rs:160-199, src/cortex/dendrites.rs:55-75,
                                     src/cortex/tufts.rs:85-101
  PyramidalLayer tuft roles          src/cortex/pyramidals.rs:84-122
  control layer order                src/cortex/control_cell_layer.rs:21
  role (cycle) order                 src/cortex/cortical_area.rs:31,601-613
  input filter chains                src/cortex/axon_space.rs:338-412

The state-slab layout (every buffer 256-byte aligned, in a fixed order) is
this project's; it is restated here from its definition (axons; per data
layer the six synapse arrays, the five dendrite arrays, for pyramidal layers
the eight cell-tuft arrays and the cell states and flags, then the cell
energies and activities, and with regrowth on one key-0 byte per dendrite;
then each filter's input buffer). tests/test_oracle.py checks that this
resolver and bm_plan_resolve agree byte for byte on every scheme the tests
use. Only the structure definitions of bismit_b200._ffi are used (no native
code is loaded).
"""
from bismit_b200 import _ffi as F

UINT64_MAX = 2 ** 64 - 1
NO_BUF = UINT64_MAX


class PlanError(ValueError):
    pass


def calc_scale(src_dim, tar_dim):
    """calc_scale, src/cmn/slice_dims.rs:201-224 (scales in 1/16ths)."""
    src, tar = src_dim * 1024, tar_dim * 1024
    if tar == 0:
        raise PlanError("Target area dimension cannot be zero.")
    incr = 1 if tar < 16 else tar // 16
    s = src // incr
    if s == 0:
        raise PlanError("Source area dimension cannot be zero.")
    if s > 255:
        raise PlanError("Source area cannot have a dimension more than 16 times target area dimension.")
    return s


def slice_dims(area_v, area_u, src, topo):
    """SliceDims::new, src/cmn/slice_dims.rs:20-94: (v_size, u_size, v_scale,
    u_scale, v_mid, u_mid) of one slice of a layer with topology `topo`,
    delivered from source `src` (None: a local layer of the area's dims)."""
    if topo in (F.BM_TOPO_SPATIAL, F.BM_TOPO_NONE):
        if src is not None:
            return (src.v_size, src.u_size, calc_scale(src.v_size, area_v), calc_scale(src.u_size, area_u), 0, 0)
        return (area_v, area_u, 16, 16, 0, 0)
    if topo == F.BM_TOPO_NONSPATIAL:
        v = src.v_size if src is not None else area_v
        u = src.u_size if src is not None else area_u
        if src is not None and (v > 255 or u > 255):
            raise PlanError("Dimensions size for horizontal layers may not exceed 255.")
        return (v, u, 0, 0, v // 2, u // 2)
    raise PlanError("unknown axon topology %d" % topo)


def gen_syn_offs(radius, vs, us):
    """gen_syn_offs, src/map/syn_src.rs:47-149: the hexagon of (v, u)
    offsets within `radius`, scaled by (vs, us) sixteenths."""
    if radius < 0:
        raise PlanError("synapse reach must be >= 0")
    v_rad, u_rad = (radius * vs) >> 4, (radius * us) >> 4
    if max(v_rad, u_rad) > 127:
        raise PlanError("scaled synapse reach exceeds 127")

    def cdiv(a, b):   # Rust's integer division truncates toward zero
        q = abs(a) // abs(b)
        return q if (a >= 0) == (b >= 0) else -q

    out = []
    for vo in range(-v_rad, v_rad + 1):
        a, b = max(-v_rad, -vo - v_rad), min(v_rad, -vo + v_rad)
        uz = cdiv(a * (us << 3), vs << 3)
        un = cdiv(b * (us << 3), vs << 3) + 1
        for uo in range(uz, un):
            if not (-127 <= vo <= 127 and -127 <= uo <= 127):
                raise PlanError("Calculated offsets are outside valid radius range")
            out.append((vo, uo))
    return out


def _align(x, a=256):
    return (x + a - 1) // a * a


def resolve(desc, seed):
    """The bm_area_plan of `desc` (a bismit_b200._ffi.bm_area_desc); raises
    PlanError where bismit's map code (or this path's limits) refuses it."""
    D = desc
    P = F.bm_area_plan()
    if D.n_layers == 0 or D.n_layers > F.BM_MAX_LAYERS:
        raise PlanError("n_layers must be 1..%d" % F.BM_MAX_LAYERS)
    if not (0 < D.v_size <= 4096 and 0 < D.u_size <= 4096):
        raise PlanError("area dims must be 1..4096")
    P.area_id, P.v_size, P.u_size, P.settings, P.rnd_seed = D.area_id, D.v_size, D.u_size, D.settings, seed

    # ---- slices (LayerMap::new + SliceMap::new): layer order, each
    # input source's slices in source order ----
    slices = []   # (layer, v_size, u_size, v_scale, u_scale, v_mid, u_mid)
    slc_start, slc_count, chains = [], [], []
    for l in range(D.n_layers):
        Ld = D.layers[l]
        for k in range(l):
            if Ld.name == D.layers[k].name:
                raise PlanError("duplicate layer name %r" % Ld.name)
        slc_start.append(len(slices))
        if Ld.axon_domain == F.BM_DOM_INPUT:
            if Ld.kind != F.BM_LYR_AXONAL:
                raise PlanError("Input layers must be 'AxonTopology::Axonal'.")
            frame_off = 0
            for s in range(Ld.n_input_srcs):
                S = Ld.input_srcs[s]
                if S.v_size == 0 or S.u_size == 0:
                    raise PlanError("input source dims are zero")
                if S.axon_topology != Ld.axon_topology:
                    if not (S.axon_topology == F.BM_TOPO_SPATIAL and Ld.axon_topology == F.BM_TOPO_NONSPATIAL):
                        raise PlanError("Layers may only convert from Spatial -> Nonspatial")
                    if S.v_size > 254 or S.u_size > 254:
                        raise PlanError("Nonspatial layer sources must be at most 254v x 254u.")
                if S.n_filters:
                    if S.n_filters > F.BM_MAX_FILTERS:
                        raise PlanError("too many filters")
                    if any(S.filters[k] != F.BM_FILTER_RETINA for k in range(S.n_filters)):
                        raise PlanError("unknown filter")
                    chains.append((l, frame_off, len(slices), S.depth, S.v_size, S.u_size,
                                   [S.filters[k] for k in range(S.n_filters)]))
                for _ in range(S.depth):
                    d = slice_dims(D.v_size, D.u_size, S, Ld.axon_topology)
                    slices.append((l,) + d)
                    frame_off += d[0] * d[1]
        else:
            for _ in range(max(Ld.depth, 0)):
                slices.append((l,) + slice_dims(D.v_size, D.u_size, None, Ld.axon_topology))
        slc_count.append(len(slices) - slc_start[l])
    if len(slices) > 255:
        raise PlanError("more than 255 axon slices")
    axons = 0
    for i, (l, vsz, usz, vsc, usc, vmid, umid) in enumerate(slices):
        P.slc_axn_idz[i], P.slc_v_size[i], P.slc_u_size[i] = axons, vsz, usz
        P.slc_v_scale[i], P.slc_u_scale[i], P.slc_v_mid[i], P.slc_u_mid[i], P.slc_layer[i] = vsc, usc, vmid, umid, l
        axons += vsz * usz
    P.n_slices, P.n_axons = len(slices), axons

    # ---- data (cellular) layers: index spaces, tuft roles, source pools ----
    data_idx = {}
    for l in range(D.n_layers):
        if D.layers[l].kind in (F.BM_LYR_SPINY_STELLATE, F.BM_LYR_PYRAMIDAL):
            data_idx[l] = len(data_idx)
    P.n_layers = len(data_idx)
    for l, di in data_idx.items():
        Ld = D.layers[l]
        L = P.layers[di]
        L.layer_id, L.kind, L.tags, L.depth = l, Ld.kind, Ld.tags, slc_count[l]
        if L.depth == 0:
            raise PlanError("cellular layer has depth 0")
        if Ld.axon_domain == F.BM_DOM_INPUT:
            raise PlanError("cellular layers cannot be input layers")
        L.base_axn_slc, L.axn_idz = slc_start[l], P.slc_axn_idz[slc_start[l]]
        L.v_size, L.u_size = D.v_size, D.u_size
        cells = D.v_size * D.u_size * L.depth
        if cells > 1 << 24:
            raise PlanError("more than 2^24 cells")
        L.cells = cells
        if not 1 <= Ld.n_tufts <= F.BM_MAX_TUFTS:
            raise PlanError("n_tufts must be 1..%d" % F.BM_MAX_TUFTS)
        if Ld.kind == F.BM_LYR_SPINY_STELLATE and Ld.n_tufts != 1:
            raise PlanError("spiny stellate layers have exactly one tuft")
        L.n_tufts = Ld.n_tufts
        syn_ttl = den_ttl = 0
        roles = set()
        for t in range(Ld.n_tufts):
            Td, T = Ld.tufts[t], L.tufts[t]
            if Td.dens_per_tft == 0 or Td.syns_per_den == 0:
                raise PlanError("TuftDims::new: dens_per_tft and syns_per_den must be > 0.")
            if Td.dens_per_tft > 256 or Td.syns_per_den > 4096 or Td.max_active_dens_l2 > 23:
                raise PlanError("tuft dims beyond this path's limits")
            T.tft_id, T.den_class, T.den_kind = t, Td.den_class, Td.den_kind
            T.dens_per_tft, T.syns_per_den = Td.dens_per_tft, Td.syns_per_den
            T.syns_per_tft = Td.dens_per_tft * Td.syns_per_den
            T.max_active_dens_l2 = Td.max_active_dens_l2
            T.den_threshold = 0 if Td.thresh_init < 0 else Td.thresh_init
            T.syn_idz, T.den_idz, T.cel_idz = syn_ttl, den_ttl, t * cells
            syn_ttl += cells * T.syns_per_tft
            den_ttl += cells * T.dens_per_tft
            if Ld.kind == F.BM_LYR_PYRAMIDAL:
                role = (Td.den_class, Td.den_kind)
                if role in roles:
                    raise PlanError("two tufts of one role")
                roles.add(role)
                if role == (F.BM_DEN_BASAL, F.BM_DEN_PROXIMAL):
                    L.bsl_prx_tft_id, flag = t, 1
                elif role == (F.BM_DEN_BASAL, F.BM_DEN_DISTAL):
                    L.bsl_dst_tft_id, flag = t, 2
                elif role == (F.BM_DEN_APICAL, F.BM_DEN_DISTAL):
                    L.apc_dst_tft_id, flag = t, 4
                else:
                    raise PlanError("apical proximal tufts are unimplemented in bismit")
                L.enabled_tft_flags |= flag
            # Source pool: every source layer's slices, repeated `prevalence`
            # times, in source order; the distinct slices sorted by id, each
            # with the reach of its last mention (a BTreeMap).
            if not 1 <= Td.n_src <= F.BM_MAX_SRC_LAYERS:
                raise PlanError("n_src must be 1..%d" % F.BM_MAX_SRC_LAYERS)
            pool, reach_of = [], {}
            for s in range(Td.n_src):
                S = Td.src[s]
                if not 0 <= S.layer_idx < D.n_layers:
                    raise PlanError("source layer index out of range")
                if S.prevalence == 0:
                    raise PlanError("Tuft source layer definitions must have a prevalence of at least one.")
                if not -128 <= S.syn_reach <= 127:
                    raise PlanError("syn_reach must fit an i8")
                ids = [slc_start[S.layer_idx] + k for k in range(slc_count[S.layer_idx])]
                pool += [(sid, S.syn_reach) for _ in range(S.prevalence) for sid in ids]
                for sid in ids:
                    reach_of[sid] = S.syn_reach
            if not pool:
                raise PlanError("Synapse source resolution error: no source layers")
            if len(pool) > F.BM_MAX_SRC_SLICES:
                raise PlanError("source pool larger than %d slices" % F.BM_MAX_SRC_SLICES)
            T.n_src = len(pool)
            for k, (sid, r) in enumerate(pool):
                T.src_slc_ids[k], T.src_reaches[k] = sid, r
            poss = 0
            for k, sid in enumerate(sorted(reach_of)):
                r = reach_of[sid]
                T.src_uniq_slc_ids[k], T.src_uniq_reaches[k] = sid, r
                if P.slc_v_scale[sid] == 0 and P.slc_u_scale[sid] == 0:
                    if P.slc_v_size[sid] & 1:
                        raise PlanError("Nonspatial slices must have u and v sizes evenly divisible by 2.")
                    poss_k = P.slc_v_size[sid] * P.slc_u_size[sid] * len(pool)
                else:
                    poss_k = len(gen_syn_offs(r, P.slc_v_scale[sid], P.slc_u_scale[sid])) * len(pool)
                if poss and poss != poss_k:
                    raise PlanError("source slices offer different numbers of offset values")
                poss = poss_k
            T.n_src_uniq = len(reach_of)
            if poss < T.syns_per_den:
                raise PlanError("not enough possible synapse source offset values")
        if syn_ttl >= 1 << 32:
            raise PlanError("2^32 or more synapses in one layer")
        L.n_syns, L.n_dens, L.n_celtfts = syn_ttl, den_ttl, cells * L.n_tufts

    # ---- control layers, in (host, exe_order) order ----
    for l in range(D.n_layers):
        Ld = D.layers[l]
        if Ld.kind < F.BM_LYR_CTRL_INHIB_BASKET:
            continue
        if Ld.host_layer_idx not in data_idx:
            raise PlanError("control layer host must be a cellular data layer")
        H = P.layers[data_idx[Ld.host_layer_idx]]
        ctrls = [H.ctrl[k] for k in range(H.n_ctrl)]
        if any(c.exe_order == Ld.exe_order for c in ctrls):
            raise PlanError("Duplicate control cell layer address / order index")
        if H.n_ctrl >= F.BM_MAX_CTRL:
            raise PlanError("too many control layers on one host")
        if Ld.kind in (F.BM_LYR_CTRL_INHIB_BASKET, F.BM_LYR_CTRL_SMOOTHER) and Ld.field_radius > 127:
            raise PlanError("field_radius must be <= 127")
        new = (Ld.kind, Ld.exe_order, Ld.field_radius, l)
        rows = [(c.kind, c.exe_order, c.field_radius, c.layer_id) for c in ctrls]
        pos = len(rows)
        while pos > 0 and rows[pos - 1][1] > Ld.exe_order:
            pos -= 1
        rows.insert(pos, new)
        for k, (kind, order, radius, lid) in enumerate(rows):
            H.ctrl[k].kind, H.ctrl[k].exe_order, H.ctrl[k].field_radius, H.ctrl[k].layer_id = kind, order, radius, lid
        H.n_ctrl = len(rows)

    # ---- input and output ranges ----
    for l in range(D.n_layers):
        if slc_count[l] == 0:
            continue
        Ld = D.layers[l]
        n = sum(P.slc_v_size[slc_start[l] + k] * P.slc_u_size[slc_start[l] + k] for k in range(slc_count[l]))
        io = (l, P.slc_axn_idz[slc_start[l]], n)
        if Ld.axon_domain == F.BM_DOM_INPUT:
            if P.n_inputs >= F.BM_MAX_IO:
                raise PlanError("too many input layers")
            P.inputs[P.n_inputs].layer_idx, P.inputs[P.n_inputs].axn_idz, P.inputs[P.n_inputs].len = io
            P.n_inputs += 1
        elif Ld.axon_domain == F.BM_DOM_OUTPUT:
            if P.n_outputs >= F.BM_MAX_IO:
                raise PlanError("too many output layers")
            P.outputs[P.n_outputs].layer_idx, P.outputs[P.n_outputs].axn_idz, P.outputs[P.n_outputs].len = io
            P.n_outputs += 1

    # ---- input filter chains ----
    for (l, frame_off, tar, depth, vsz, usz, filters) in chains:
        inp = [i for i in range(P.n_inputs) if P.inputs[i].layer_idx == l]
        if not inp:
            raise PlanError("filter chain on a layer that is not an input layer")
        if depth == 0:
            raise PlanError("filter chain on a source of depth 0")
        if vsz % 8 or usz % 8:
            raise PlanError("filter chain source dims are not multiples of 8 (1 x 8 x 8 work-groups)")
        for k in range(depth):
            if P.slc_v_size[tar + k] != vsz or P.slc_u_size[tar + k] != usz:
                raise PlanError("filter chain target slice dims differ from the source's")
        if len(filters) > 1:
            for k in range(depth):
                if P.slc_axn_idz[k] + vsz * usz > depth * vsz * usz:
                    raise PlanError("an inner filter would write past its buffer")
        if P.n_filter_chains >= F.BM_MAX_IO:
            raise PlanError("too many filter chains")
        c = P.filter_chains[P.n_filter_chains]
        c.input, c.frame_off, c.tar_slc, c.depth, c.v_size, c.u_size = inp[-1], frame_off, tar, depth, vsz, usz
        c.n_filters = len(filters)
        for k, f in enumerate(filters):
            c.filters[k] = f
        P.n_filter_chains += 1

    # ---- cycle order: focus, spatial, temporal, motor layers ----
    used = set()
    for role in (F.BM_TAG_FOCUS, F.BM_TAG_SPATIAL, F.BM_TAG_TEMPORAL, F.BM_TAG_MOTOR):
        for i in range(P.n_layers):
            if P.layers[i].tags & role and i not in used:
                used.add(i)
                P.cycle_order[P.n_cycle_order] = i
                P.n_cycle_order += 1

    # ---- state slab ----
    off = _align(P.n_axons)
    P.axon_off = 0
    total = 0
    for i in range(P.n_layers):
        L = P.layers[i]
        for k in range(F.BM_BUF_COUNT):
            L.buf_off[k], L.buf_len[k] = NO_BUF, 0

        def put(k, n):
            nonlocal off
            L.buf_off[k], L.buf_len[k] = off, n
            off = _align(off + n)

        for name in ("syn_states", "syn_strengths", "syn_src_slc_ids", "syn_src_col_v_offs", "syn_src_col_u_offs",
                     "syn_flag_sets"):
            put(F.BUF[name], L.n_syns)
        for name in ("den_states_raw", "den_states", "den_energies", "den_activities", "den_thresholds"):
            put(F.BUF[name], L.n_dens)
        if L.kind == F.BM_LYR_PYRAMIDAL:
            for name in ("tft_prev_best_den_ids", "tft_prev_best_den_states_raw", "tft_prev_best_den_states",
                         "tft_prev_states", "tft_best_den_ids", "tft_best_den_states_raw", "tft_best_den_states",
                         "tft_states"):
                put(F.BUF[name], L.n_celtfts)
            put(F.BUF["cel_states"], L.cells)
            put(F.BUF["cel_flag_sets"], L.cells)
        put(F.BUF["cel_energies"], L.cells)
        put(F.BUF["cel_activities"], L.cells)
        if not P.settings & F.BM_SET_DISABLE_REGROWTH:
            put(F.BUF["den_src_key0"], L.n_dens)
        total += L.n_syns
    for i in range(P.n_filter_chains):
        c = P.filter_chains[i]
        for k in range(c.n_filters):
            c.buf_off[k] = off
            off = _align(off + c.depth * c.v_size * c.u_size)
    P.slab_bytes = off
    P.n_syns_total = total
    return P
