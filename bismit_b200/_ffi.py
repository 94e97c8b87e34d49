"""ctypes bindings of the C ABI in include/bismit_b200.h.

The structures below mirror the header field for field. Loading fails loudly
when the native library has not been built: there is no fallback path.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbismit_b200.so")

# ---------------------------------------------------------------- constants --
BM_OK, BM_ERR_INVALID, BM_ERR_OOM, BM_ERR_CUDA, BM_ERR_TIMEOUT, BM_ERR_UNSUPPORTED, BM_ERR_NO_DEVICE = range(7)
BM_MAX_SLICES = 256
BM_MAX_LAYERS = 16
BM_MAX_TUFTS = 4
BM_MAX_SRC_LAYERS = 8
BM_MAX_SRC_SLICES = 32
BM_MAX_CTRL = 4
BM_MAX_IO = 8
BM_MAX_FILTERS = 4
BM_NAME_LEN = 32

BM_LYR_AXONAL, BM_LYR_SPINY_STELLATE, BM_LYR_PYRAMIDAL = 0, 1, 2
BM_LYR_CTRL_INHIB_BASKET, BM_LYR_CTRL_PYR_OUTPUT, BM_LYR_CTRL_INTRA_COLUMN, BM_LYR_CTRL_SMOOTHER = 3, 4, 5, 6
BM_DOM_LOCAL, BM_DOM_INPUT, BM_DOM_OUTPUT = 0, 1, 2
BM_TOPO_SPATIAL, BM_TOPO_NONSPATIAL, BM_TOPO_NONE = 0, 1, 2
BM_DEN_BASAL, BM_DEN_APICAL = 0, 1
BM_DEN_PROXIMAL, BM_DEN_DISTAL = 0, 1

BM_TAG_PRIMARY = 1 << 32
BM_TAG_SPATIAL = 1 << 36
BM_TAG_TEMPORAL = 1 << 37
BM_TAG_FOCUS = 1 << 38
BM_TAG_MOTOR = 1 << 39
BM_TAG_UNUSED = 1 << 47
BM_TAG_INPUT = 1 << 48
BM_TAG_OUTPUT = 1 << 49

BM_SET_BYPASS_INHIB = 1 << 0
BM_SET_BYPASS_FILTERS = 1 << 1
BM_SET_DISABLE_PYRS = 1 << 2
BM_SET_DISABLE_SSCS = 1 << 3
BM_SET_DISABLE_MCOLS = 1 << 4
BM_SET_DISABLE_REGROWTH = 1 << 5
BM_SET_DISABLE_LEARNING = 1 << 6

BM_INIT_STRENGTH_ZERO = 1 << 0
BM_INIT_NO_UNIQUE = 1 << 1
BM_PATH_FUSED, BM_PATH_PLAIN = 0, 1
BM_FILTER_RETINA = 1

BUF_NAMES = [
    "syn_states", "syn_strengths", "syn_src_slc_ids", "syn_src_col_v_offs", "syn_src_col_u_offs",
    "syn_flag_sets", "den_states_raw", "den_states", "den_energies", "den_activities", "den_thresholds",
    "tft_prev_best_den_ids", "tft_prev_best_den_states_raw", "tft_prev_best_den_states", "tft_prev_states",
    "tft_best_den_ids", "tft_best_den_states_raw", "tft_best_den_states", "tft_states",
    "cel_energies", "cel_activities", "cel_states", "cel_flag_sets", "den_src_key0",
]
BM_BUF_COUNT = len(BUF_NAMES)
BUF = {n: i for i, n in enumerate(BUF_NAMES)}
BM_BUF_AXON_STATES = 64
BM_ALL_LAYERS = 0xFFFFFFFF
SIGNED_BUFS = {"syn_strengths", "syn_src_col_v_offs", "syn_src_col_u_offs"}

BM_RND_DEN_CYCLE, BM_RND_INHIB, BM_RND_SSC_MTP, BM_RND_TFT_DST_MTP = 1, 2, 3, 4


# --------------------------------------------------------------- structures --
class bm_src_layer_desc(C.Structure):
    _fields_ = [("layer_idx", C.c_int32), ("syn_reach", C.c_int32), ("prevalence", C.c_uint32)]


class bm_tuft_desc(C.Structure):
    _fields_ = [
        ("den_class", C.c_uint32), ("den_kind", C.c_uint32), ("dens_per_tft", C.c_uint32),
        ("syns_per_den", C.c_uint32), ("max_active_dens_l2", C.c_uint32), ("thresh_init", C.c_int64),
        ("n_src", C.c_uint32), ("src", bm_src_layer_desc * BM_MAX_SRC_LAYERS),
    ]


class bm_input_src_desc(C.Structure):
    _fields_ = [("v_size", C.c_uint32), ("u_size", C.c_uint32), ("depth", C.c_uint32), ("axon_topology", C.c_uint32),
                ("n_filters", C.c_uint32), ("filters", C.c_uint32 * BM_MAX_FILTERS)]


class bm_layer_desc(C.Structure):
    _fields_ = [
        ("name", C.c_char * BM_NAME_LEN), ("tags", C.c_uint64), ("kind", C.c_uint32), ("depth", C.c_int32),
        ("axon_topology", C.c_uint32), ("axon_domain", C.c_uint32), ("n_input_srcs", C.c_uint32),
        ("input_srcs", bm_input_src_desc * BM_MAX_IO), ("host_layer_idx", C.c_int32),
        ("field_radius", C.c_uint32), ("exe_order", C.c_uint32), ("n_tufts", C.c_uint32),
        ("tufts", bm_tuft_desc * BM_MAX_TUFTS),
    ]


class bm_area_desc(C.Structure):
    _fields_ = [
        ("area_id", C.c_uint32), ("v_size", C.c_uint32), ("u_size", C.c_uint32), ("n_layers", C.c_uint32),
        ("layers", bm_layer_desc * BM_MAX_LAYERS), ("settings", C.c_uint32), ("init_flags", C.c_uint32),
        ("exec_path", C.c_uint32),
    ]


class bm_tuft_plan(C.Structure):
    _fields_ = [
        ("tft_id", C.c_uint32), ("den_class", C.c_uint32), ("den_kind", C.c_uint32),
        ("dens_per_tft", C.c_uint32), ("syns_per_den", C.c_uint32), ("syns_per_tft", C.c_uint32),
        ("max_active_dens_l2", C.c_uint32), ("den_threshold", C.c_uint32),
        ("syn_idz", C.c_uint64), ("den_idz", C.c_uint64), ("cel_idz", C.c_uint64),
        ("n_src", C.c_uint32), ("src_slc_ids", C.c_uint8 * BM_MAX_SRC_SLICES),
        ("src_reaches", C.c_int8 * BM_MAX_SRC_SLICES), ("n_src_uniq", C.c_uint32),
        ("src_uniq_slc_ids", C.c_uint8 * BM_MAX_SRC_SLICES), ("src_uniq_reaches", C.c_int8 * BM_MAX_SRC_SLICES),
    ]


class bm_ctrl_plan(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("exe_order", C.c_uint32), ("field_radius", C.c_uint32), ("layer_id", C.c_uint32)]


class bm_layer_plan(C.Structure):
    _fields_ = [
        ("layer_id", C.c_uint32), ("kind", C.c_uint32), ("tags", C.c_uint64), ("depth", C.c_uint32),
        ("base_axn_slc", C.c_uint32), ("axn_idz", C.c_uint32), ("v_size", C.c_uint32), ("u_size", C.c_uint32),
        ("cells", C.c_uint32), ("n_tufts", C.c_uint32), ("tufts", bm_tuft_plan * BM_MAX_TUFTS),
        ("n_syns", C.c_uint64), ("n_dens", C.c_uint64), ("n_celtfts", C.c_uint64),
        ("enabled_tft_flags", C.c_uint32), ("bsl_prx_tft_id", C.c_uint32), ("bsl_dst_tft_id", C.c_uint32),
        ("apc_dst_tft_id", C.c_uint32), ("n_ctrl", C.c_uint32), ("ctrl", bm_ctrl_plan * BM_MAX_CTRL),
        ("buf_off", C.c_uint64 * BM_BUF_COUNT), ("buf_len", C.c_uint64 * BM_BUF_COUNT),
    ]


class bm_io_plan(C.Structure):
    _fields_ = [("layer_idx", C.c_uint32), ("axn_idz", C.c_uint32), ("len", C.c_uint32)]


class bm_filter_chain_plan(C.Structure):
    _fields_ = [
        ("input", C.c_uint32), ("frame_off", C.c_uint32), ("tar_slc", C.c_uint32), ("depth", C.c_uint32),
        ("v_size", C.c_uint32), ("u_size", C.c_uint32), ("n_filters", C.c_uint32),
        ("filters", C.c_uint32 * BM_MAX_FILTERS), ("buf_off", C.c_uint64 * BM_MAX_FILTERS),
    ]


class bm_area_plan(C.Structure):
    _fields_ = [
        ("area_id", C.c_uint32), ("v_size", C.c_uint32), ("u_size", C.c_uint32), ("settings", C.c_uint32),
        ("n_slices", C.c_uint32),
        ("slc_axn_idz", C.c_uint32 * BM_MAX_SLICES), ("slc_v_size", C.c_uint32 * BM_MAX_SLICES),
        ("slc_u_size", C.c_uint32 * BM_MAX_SLICES), ("slc_v_scale", C.c_uint32 * BM_MAX_SLICES),
        ("slc_u_scale", C.c_uint32 * BM_MAX_SLICES), ("slc_v_mid", C.c_uint32 * BM_MAX_SLICES),
        ("slc_u_mid", C.c_uint32 * BM_MAX_SLICES), ("slc_layer", C.c_uint32 * BM_MAX_SLICES),
        ("n_axons", C.c_uint32), ("axon_off", C.c_uint64),
        ("n_inputs", C.c_uint32), ("inputs", bm_io_plan * BM_MAX_IO),
        ("n_outputs", C.c_uint32), ("outputs", bm_io_plan * BM_MAX_IO),
        ("n_layers", C.c_uint32), ("layers", bm_layer_plan * BM_MAX_LAYERS),
        ("n_cycle_order", C.c_uint32), ("cycle_order", C.c_uint32 * BM_MAX_LAYERS),
        ("slab_bytes", C.c_uint64), ("n_syns_total", C.c_uint64), ("rnd_seed", C.c_uint64),
        ("n_filter_chains", C.c_uint32), ("filter_chains", bm_filter_chain_plan * BM_MAX_IO),
    ]


# ------------------------------------------------------------------ loading --
_lib = None


class BismitError(RuntimeError):
    """A non-zero status from the C ABI (the CmnError of the reference)."""

    def __init__(self, code, msg):
        super().__init__("bismit_b200 error %d: %s" % (code, msg))
        self.code = code


class bm_server_stats(C.Structure):
    _fields_ = [("ticks", C.c_uint64), ("frames", C.c_uint64), ("batch_rebuilds", C.c_uint64),
                ("syn_cycles", C.c_double), ("busy_s", C.c_double), ("rebuild_s", C.c_double),
                ("admit_s", C.c_double), ("gpu_s", C.c_double), ("span_s", C.c_double),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
                ("used_bytes", C.c_uint64), ("budget_bytes", C.c_uint64),
                ("resident", C.c_uint32), ("waiting", C.c_uint32), ("failed", C.c_uint32),
                ("rebuild_drains", C.c_uint64), ("capture_s", C.c_double),
                ("tick_p99_ms", C.c_double), ("tick_max_ms", C.c_double), ("tick_max_no", C.c_uint64),
                ("tick_max_members", C.c_uint32), ("tick_max_what", C.c_uint32),
                ("tick_max_queue_ms", C.c_double), ("tick_max_builder", C.c_uint32), ("pad0", C.c_uint32),
                ("tick_max_builder_ms", C.c_double)]


# bm_server_stats.tick_max_what bits
BM_TICK_FIRST, BM_TICK_REBUILD, BM_TICK_DRAIN, BM_TICK_CAPTURE = 1, 2, 4, 8
# bm_server_stats.tick_max_builder bits
BM_BUILDER_BUILD, BM_BUILDER_BATCH, BM_BUILDER_DEVICE_BUFFER, BM_BUILDER_AREA_FREE, BM_BUILDER_OUTPUT_FREE = \
    1, 2, 4, 8, 16


class bm_tuft_form(C.Structure):
    _fields_ = [("fused", C.c_uint32), ("tiled", C.c_uint32), ("consumer", C.c_uint32),
                ("sources_outside", C.c_uint32), ("flags_foreign", C.c_uint32), ("tile_w", C.c_uint32),
                ("tile_h", C.c_uint32), ("stages", C.c_uint32), ("grid", C.c_uint32), ("smem", C.c_uint32),
                ("footprint_tma", C.c_uint32)]


def lib():
    """Returns the loaded native library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("bismit_b200 native library missing (%s): run `python -m bismit_b200.build`" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    vp, u32, u64, i32, sz = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_size_t
    P = C.POINTER
    sigs = {
        "bm_last_error": (C.c_char_p, []),
        "bm_version": (C.c_char_p, []),
        "bm_ctx_create": (C.c_int, [C.c_int, u32, P(vp)]),
        "bm_ctx_destroy": (C.c_int, [vp]),
        "bm_ctx_set_stream": (C.c_int, [vp, vp]),
        "bm_ctx_use_own_stream": (C.c_int, [vp]),
        "bm_ctx_synchronize": (C.c_int, [vp]),
        "bm_area_create": (C.c_int, [vp, P(bm_area_desc), u64, P(vp)]),
        "bm_area_destroy": (C.c_int, [vp]),
        "bm_area_get_plan": (C.c_int, [vp, P(bm_area_plan)]),
        "bm_plan_resolve": (C.c_int, [P(bm_area_desc), u64, P(bm_area_plan)]),
        "bm_area_write_input": (C.c_int, [vp, u32, vp, sz]),
        "bm_area_write_input_device": (C.c_int, [vp, u32, vp, sz]),
        "bm_area_cycle": (C.c_int, [vp, u32]),
        "bm_area_cycle_frames_device": (C.c_int, [vp, vp, sz, u32]),
        "bm_area_read_output": (C.c_int, [vp, u32, vp, sz]),
        "bm_area_read": (C.c_int, [vp, u32, u32, u64, vp, u64]),
        "bm_area_write": (C.c_int, [vp, u32, u32, u64, vp, u64]),
        "bm_area_read_slab": (C.c_int, [vp, vp, u64]),
        "bm_area_side_steps": (C.c_int, [vp, P(u32)]),
        "bm_area_front_steps": (C.c_int, [vp, P(u32)]),
        "bm_sampler_create": (C.c_int, [vp, u32, u32, C.c_int, P(vp)]),
        "bm_sampler_destroy": (C.c_int, [vp]),
        "bm_sampler_len": (C.c_int, [vp, P(u64)]),
        "bm_sampler_set_backpressure": (C.c_int, [vp, C.c_int, P(C.c_int)]),
        "bm_sampler_set_timeout": (C.c_int, [vp, u32]),
        "bm_sampler_recv": (C.c_int, [vp, C.c_int, vp, u64, P(u64), P(C.c_int)]),
        "bm_sampler_stats": (C.c_int, [vp, P(u64), P(u64)]),
        "bm_encode_images": (C.c_int, [vp, vp, u32, u32, u32, C.c_float, vp, u64, u32, u32]),
        "bm_encode_hex_mold": (C.c_int, [vp, C.c_int32, u32, u32, vp, u32, u32]),
        "bm_encode_scalar": (C.c_int, [vp, vp, u32, C.c_float, C.c_float, u64, vp, u64, u32, u32]),
        "bm_encode_scalar_glyph": (C.c_int, [vp, vp, u32, C.c_float, C.c_float, vp, u64, u32, u32]),
        "bm_sdr_writer_create": (C.c_int, [vp, C.c_float, C.c_float, C.c_float, u32, u32, u64, P(vp)]),
        "bm_sdr_writer_destroy": (C.c_int, [vp]),
        "bm_sdr_writer_info": (C.c_int, [vp, P(u32), P(u32), P(u32)]),
        "bm_sdr_writer_waypoints": (C.c_int, [vp, vp, u64]),
        "bm_sdr_writer_encode": (C.c_int, [vp, vp, u32, vp, u64]),
        "bm_area_write_slab": (C.c_int, [vp, vp, u64]),
        "bm_area_get_cycle": (C.c_int, [vp, P(u64)]),
        "bm_area_set_cycle": (C.c_int, [vp, u64]),
        "bm_area_slab_ptr": (C.c_int, [vp, P(vp)]),
        "bm_area_sources_changed": (C.c_int, [vp, u32]),
        "bm_area_device_errors": (C.c_int, [vp, P(u32)]),
        "bm_area_tuft_form": (C.c_int, [vp, u32, u32, P(bm_tuft_form)]),
        "bm_area_clear_errors": (C.c_int, [vp]),
        "bm_area_deliver_tract": (C.c_int, [vp, u32, vp, u32, u64]),
        "bm_area_axons_touched": (C.c_int, [vp]),
        "bm_area_set_wait_limit": (C.c_int, [vp, u32]),
        "bm_area_inject_stall": (C.c_int, [vp, u32]),
        "bm_area_set_profiling": (C.c_int, [vp, C.c_int]),
        "bm_area_get_profile": (C.c_int, [vp, u32, P(C.c_char_p), P(u64), P(C.c_double), P(u32)]),
        "bm_area_reset_profile": (C.c_int, [vp]),
        "bm_area_launches_per_cycle": (C.c_int, [vp, P(u32)]),
        "bm_tuft_cycle_static": (C.c_int, [P(bm_area_plan), u32, u32, vp, u64, vp, vp]),
        "bm_batch_create": (C.c_int, [vp, P(vp), u32, P(vp)]),
        "bm_batch_destroy": (C.c_int, [vp]),
        "bm_batch_set_graph": (C.c_int, [vp, C.c_int]),
        "bm_batch_cycle": (C.c_int, [vp, u32]),
        "bm_batch_frame_bytes": (C.c_int, [vp, P(u64)]),
        "bm_batch_connect": (C.c_int, [vp, u32, u32, u32, u32, u64]),
        "bm_batch_cycle_frames_device": (C.c_int, [vp, vp, u32]),
        "bm_batch_launches_per_cycle": (C.c_int, [vp, P(u32)]),
        "bm_batch_device_errors": (C.c_int, [vp, P(u32)]),
        "bm_batch_autotune": (C.c_int, [vp, C.c_char_p, P(u32)]),
        "bm_batch_set_profiling": (C.c_int, [vp, C.c_int]),
        "bm_batch_get_profile": (C.c_int, [vp, u32, P(u32), P(u32), P(u32), P(u32), P(u64), P(C.c_double), P(u32)]),
        "bm_batch_reset_profile": (C.c_int, [vp]),
        "bm_server_create": (C.c_int, [vp, u64, P(vp)]),
        "bm_server_destroy": (C.c_int, [vp]),
        "bm_server_open": (C.c_int, [vp, P(bm_area_desc), u64, P(u32)]),
        "bm_server_submit": (C.c_int, [vp, u32, vp, sz, u32]),
        "bm_server_close": (C.c_int, [vp, u32]),
        "bm_server_cancel": (C.c_int, [vp, u32]),
        "bm_server_tick": (C.c_int, [vp, P(u32)]),
        "bm_server_drain": (C.c_int, [vp]),
        "bm_server_read_output": (C.c_int, [vp, u32, vp, sz, P(u64)]),
        "bm_server_session_area": (C.c_int, [vp, u32, P(vp)]),
        "bm_server_get_stats": (C.c_int, [vp, P(bm_server_stats)]),
        "bm_server_reset_stats": (C.c_int, [vp]),
        "bm_rnd": (i32, [u64, u32, u32, u32, u32, u64]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(rc):
    if rc != BM_OK:
        raise BismitError(rc, lib().bm_last_error().decode(errors="replace"))
    return rc
