"""CPU oracle loaders (TEST INFRASTRUCTURE).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package. It never runs inside the product library.

  load_port()  -> oracle/libbm_oracle.so, the C restatement (bm_oracle.c)
  load_ref()   -> oracle/_ref/libbm_ref.so, bismit's own cl/*.cl kernels compiled
                  for the CPU (None if it was not built, e.g. without a bismit
                  checkout)
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "libbm_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libbm_ref.so")
REFERENCE_CHECKOUT = os.environ.get("BISMIT_REFERENCE", "")

_port = None
_ref = None


def build(ref=True, checkout=None):
    """Builds the port, and the reference kernels when a bismit checkout is
    given (`checkout`, else $BISMIT_REFERENCE) and holds cl/."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    checkout = checkout or REFERENCE_CHECKOUT
    if ref and checkout and os.path.isdir(os.path.join(checkout, "cl")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "BISMIT=%s" % checkout], check=True)


def _plan_ptr(plan):
    from bismit_b200 import _ffi as F  # plan struct layout only
    assert isinstance(plan, F.bm_area_plan)
    return C.byref(plan)


def load_port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_PATH):
            build(ref=False)
        L = C.CDLL(PORT_PATH)
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        L.bmo_run.restype = C.c_int
        L.bmo_run.argtypes = [vp, vp, vp, u64, u32, u64, C.c_int]
        f32 = C.c_float
        L.bmo_encode_image.restype = None
        L.bmo_encode_image.argtypes = [vp, u32, u32, f32, vp, u32, u32]
        L.bmo_hex_mold.restype = C.c_int
        L.bmo_hex_mold.argtypes = [C.c_int, u32, u32, vp, u32, u32]
        L.bmo_encode_scalar.restype = C.c_int
        L.bmo_encode_scalar.argtypes = [f32, f32, f32, u64, u32, vp, u32, u32]
        L.bmo_encode_scalar_glyph.restype = C.c_int
        L.bmo_encode_scalar_glyph.argtypes = [f32, f32, f32, vp, u32, u32]
        L.bmo_sdr_waypoints.restype = C.c_int
        L.bmo_sdr_waypoints.argtypes = [f32, f32, f32, u32, u32, u64, vp]
        L.bmo_sdr_encode.restype = C.c_int
        L.bmo_sdr_encode.argtypes = [f32, f32, f32, f32, u32, vp, vp, u32]
        L.bmo_intake.restype = C.c_int
        L.bmo_intake.argtypes = [vp, vp, u32, u32, vp, u32]
        L.bmo_grow.restype = C.c_int
        L.bmo_grow.argtypes = [vp, vp, u64, u32]
        L.bmo_rnd.restype = C.c_int32
        L.bmo_rnd.argtypes = [u64, u32, u32, u32, u32, u64]
        L.bmo_gen_syn_offs.restype = C.c_int
        L.bmo_gen_syn_offs.argtypes = [C.c_int, u32, u32, vp, vp, C.c_int]
        L.bmo_axn_idx_scl.restype = u32
        L.bmo_axn_idx_scl.argtypes = [vp, C.c_uint8, u32, C.c_int8, u32, C.c_int8, C.POINTER(C.c_int)]
        L.bmo_axn_idx_vec4.restype = u32
        L.bmo_axn_idx_vec4.argtypes = [vp, C.c_uint8, C.c_int32, C.c_int8, C.c_int32, C.c_int8, C.POINTER(C.c_int)]
        _port = L
    return _port


def load_ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_PATH):
            return None
        L = C.CDLL(REF_PATH)
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        L.bmr_run.restype = C.c_int
        L.bmr_run.argtypes = [vp, vp, vp, u64, u32, u64, C.c_int]
        L.bmr_test_axn_idxs.restype = C.c_int
        L.bmr_test_axn_idxs.argtypes = [vp, u32, u32, u32, vp, vp, vp, vp]
        _ref = L
    return _ref


def _np_ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def run(plan, slab, frames=None, n_cycles=1, start_cycle=0, threads=0, impl="port"):
    """Runs n_cycles cycles on `slab` (uint8 array of plan.slab_bytes) in place.
    `frames` is None or an (n_cycles, input_len) uint8 array."""
    L = load_port() if impl == "port" else load_ref()
    if L is None:
        raise RuntimeError("the reference-kernel oracle (oracle/_ref) is not built")
    fn = L.bmo_run if impl == "port" else L.bmr_run
    assert slab.dtype == np.uint8 and slab.flags.c_contiguous and slab.size == plan.slab_bytes
    flen = 0
    if frames is not None:
        frames = np.ascontiguousarray(frames, dtype=np.uint8)
        assert frames.shape[0] >= n_cycles
        flen = frames.shape[1]
    rc = fn(C.cast(_plan_ptr(plan), C.c_void_p), _np_ptr(slab), _np_ptr(frames), flen, n_cycles, start_cycle, threads)
    if rc != 0:
        raise RuntimeError("oracle run failed (%d)" % rc)


def intake(plan, slab, input_idx, offset, data):
    """Writes `data` at byte `offset` of a frame of input `input_idx`, where
    intake puts it (a filtered source's bytes into its chain's first buffer)."""
    data = np.ascontiguousarray(data, dtype=np.uint8)
    rc = load_port().bmo_intake(C.cast(_plan_ptr(plan), C.c_void_p), _np_ptr(slab), input_idx, offset,
                                _np_ptr(data), data.size)
    if rc != 0:
        raise RuntimeError("oracle intake out of range")


def grow(plan, slab, seed, init_flags):
    rc = load_port().bmo_grow(C.cast(_plan_ptr(plan), C.c_void_p), _np_ptr(slab), seed, init_flags)
    if rc != 0:
        raise RuntimeError("oracle growth failed (%d)" % rc)


def rnd(seed, area_id, layer_id, role, tft_id, cycle):
    return load_port().bmo_rnd(seed, area_id, layer_id, role, tft_id, cycle)


def gen_syn_offs(radius, v_scale, u_scale):
    cap = 3 * 127 * 128 + 1
    v = np.zeros(cap, np.int8)
    u = np.zeros(cap, np.int8)
    n = load_port().bmo_gen_syn_offs(radius, v_scale, u_scale, _np_ptr(v), _np_ptr(u), cap)
    if n < 0:
        raise ValueError("gen_syn_offs failed")
    return v[:n].copy(), u[:n].copy()


def ref_axn_idxs(plan, depth, v_size, u_size, v_offs, u_offs):
    L = load_ref()
    if L is None:
        raise RuntimeError("oracle/_ref is not built")
    n = depth * v_size * u_size
    v = np.ascontiguousarray(v_offs, np.int8)
    u = np.ascontiguousarray(u_offs, np.int8)
    o1 = np.zeros(n, np.uint32)
    o2 = np.zeros(n, np.uint32)
    rc = L.bmr_test_axn_idxs(C.cast(_plan_ptr(plan), C.c_void_p), depth, v_size, u_size, _np_ptr(v), _np_ptr(u),
                             _np_ptr(o1), _np_ptr(o2))
    if rc != 0:
        raise RuntimeError("test_axn_idxs failed (%d)" % rc)
    return o1, o2


# ----------------------------------------------------------------- encoders --

def encode_image(image, scale_factor, v_size, u_size, target=None):
    """encode_2d_image of one (x_size, y_size)-shaped image (rows of x_size
    bytes, y_size rows) onto a v_size x u_size frame; cells outside the image
    keep `target`'s bytes (zeros when not given)."""
    img = np.ascontiguousarray(image, dtype=np.uint8)
    y_size, x_size = img.shape
    out = np.zeros(v_size * u_size, np.uint8) if target is None else np.array(target, np.uint8, copy=True)
    load_port().bmo_encode_image(_np_ptr(img), x_size, y_size, scale_factor, _np_ptr(out), v_size, u_size)
    return out


def hex_mold(radius, src_dims, v_size, u_size):
    out = np.zeros(v_size * u_size, np.uint8)
    n = load_port().bmo_hex_mold(radius, src_dims[0], src_dims[1], _np_ptr(out), v_size, u_size)
    if n < 0:
        raise ValueError("hex mold refused")
    return out, n


def encode_scalar(vals, lo, hi, seed, v_size, u_size):
    out = np.zeros((len(vals), v_size * u_size), np.uint8)
    for k, v in enumerate(vals):
        if load_port().bmo_encode_scalar(v, lo, hi, seed, k, _np_ptr(out[k]), v_size, u_size) != 0:
            raise ValueError("value %r refused" % v)
    return out


def encode_scalar_glyph(vals, lo, hi, v_size, u_size):
    out = np.zeros((len(vals), v_size * u_size), np.uint8)
    for k, v in enumerate(vals):
        if load_port().bmo_encode_scalar_glyph(v, lo, hi, _np_ptr(out[k]), v_size, u_size) != 0:
            raise ValueError("value %r refused" % v)
    return out


def sdr_waypoints(lo, hi, way_span, v_size, u_size, seed):
    n = load_port().bmo_sdr_waypoints(lo, hi, way_span, v_size, u_size, seed, None)
    if n < 0:
        raise ValueError("writer refused")
    ways = np.zeros((n, (v_size * u_size) // 48), np.uint32)
    load_port().bmo_sdr_waypoints(lo, hi, way_span, v_size, u_size, seed, _np_ptr(ways))
    return ways


def sdr_encode(vals, lo, hi, way_span, ways, length):
    out = np.zeros((len(vals), length), np.uint8)
    w = np.ascontiguousarray(ways, dtype=np.uint32)
    for k, v in enumerate(vals):
        if load_port().bmo_sdr_encode(v, lo, hi, way_span, w.shape[0], _np_ptr(w), _np_ptr(out[k]), length) != 0:
            raise ValueError("value %r refused" % v)
    return out
