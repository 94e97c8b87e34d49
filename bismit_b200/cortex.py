"""Cortex and CorticalArea: the host objects of the cortical cycle.

Mirrors the reference's drop-in surface for this path
(src/cortex/cortex.rs:37-201, src/cortex/cortical_area.rs:343-1321):
``Cortex.builder(layer_map_schemes, area_schemes).ca_settings(..).build()``,
``cortex.cycle()``, per-area ``cycle``, input intake and output, and the raw
buffer read/write/fill helpers of the reference's test traits. Every call goes
through the C ABI of the native library; errors raise BismitError.
"""
import ctypes as C
import weakref

import numpy as np

from . import _ffi as F
from .map import (AreaSchemeList, CorticalAreaSettings, LayerMapKind, LayerMapSchemeList, area_desc, area_tracts)


class _Ctx:
    def __init__(self, device=0):
        self.lib = F.lib()
        self.h = C.c_void_p()
        F.check(self.lib.bm_ctx_create(int(device), 0, C.byref(self.h)))
        self.device = device
        self._owned = []   # weak references to the areas, batches and servers made on this context

    def _adopt(self, obj):
        self._owned = [r for r in self._owned if r() is not None]
        self._owned.append(weakref.ref(obj))

    def set_stream(self, stream_ptr):
        F.check(self.lib.bm_ctx_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    def synchronize(self):
        F.check(self.lib.bm_ctx_synchronize(self.h))

    def close(self):
        """Destroys the context after everything made on it (batches and
        servers first, then areas): finalizers at interpreter exit run in no
        set order, and a handle must not outlive what it points into."""
        if self.h:
            objs = [o for o in (r() for r in self._owned) if o is not None]
            for o in objs:
                if not isinstance(o, CorticalArea):
                    o.close()
            for o in objs:
                o.close()
            self._owned = []
            self.lib.bm_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CorticalArea:
    """One cortical area on the device (CorticalArea, src/cortex/cortical_area.rs:343)."""

    def __init__(self, ctx, desc, seed, name=""):
        self.lib = F.lib()
        self.ctx = ctx
        self.name = name
        self.desc = desc
        self.h = C.c_void_p()
        F.check(self.lib.bm_area_create(ctx.h, C.byref(desc), C.c_uint64(seed), C.byref(self.h)))
        self._holders = []
        self._samplers = []
        ctx._adopt(self)
        self.plan = F.bm_area_plan()
        F.check(self.lib.bm_area_get_plan(self.h, C.byref(self.plan)))
        self.layer_names = [desc.layers[i].name.decode() for i in range(desc.n_layers)]

    # ---- structure ----
    def data_layer(self, name_or_idx):
        """Plan index of a data (cellular) layer, by scheme name or plan index."""
        if isinstance(name_or_idx, int):
            return name_or_idx
        lid = self.layer_names.index(name_or_idx)
        for i in range(self.plan.n_layers):
            if self.plan.layers[i].layer_id == lid:
                return i
        raise KeyError("%r is not a cellular layer" % name_or_idx)

    @property
    def n_syns(self):
        return int(self.plan.n_syns_total)

    @property
    def slab_bytes(self):
        return int(self.plan.slab_bytes)

    def input_len(self, idx=0):
        return int(self.plan.inputs[idx].len)

    def output_len(self, idx=0):
        return int(self.plan.outputs[idx].len)

    # ---- cycle ----
    def write_input(self, frame, idx=0):
        """AxonSpace::intake: one u8 frame into input layer `idx` (src/cortex/axon_space.rs:509)."""
        a = np.ascontiguousarray(frame, dtype=np.uint8)
        F.check(self.lib.bm_area_write_input(self.h, idx, a.ctypes.data_as(C.c_void_p), a.nbytes))

    def cycle(self, n=1):
        """CorticalArea::cycle n times (src/cortex/cortical_area.rs:716)."""
        F.check(self.lib.bm_area_cycle(self.h, int(n)))

    def cycle_frames_device(self, dev_ptr, frame_len, n):
        F.check(self.lib.bm_area_cycle_frames_device(self.h, C.c_void_p(dev_ptr), frame_len, int(n)))

    def read_output(self, idx=0):
        """AxonSpace::output: the output layer's axons (src/cortex/axon_space.rs:594)."""
        out = np.empty(self.output_len(idx), dtype=np.uint8)
        F.check(self.lib.bm_area_read_output(self.h, idx, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    # ---- raw buffers (sampler / test-trait surface) ----
    def read(self, buf, layer=0, offset=0, length=None):
        kind = F.BM_BUF_AXON_STATES if buf == "axon_states" else F.BUF[buf]
        li = 0 if kind == F.BM_BUF_AXON_STATES else self.data_layer(layer)
        if length is None:
            length = (self.plan.n_axons if kind == F.BM_BUF_AXON_STATES
                      else self.plan.layers[li].buf_len[kind]) - offset
        dt = np.int8 if buf in F.SIGNED_BUFS else np.uint8
        out = np.empty(int(length), dtype=dt)
        F.check(self.lib.bm_area_read(self.h, kind, li, int(offset), out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def write(self, buf, data, layer=0, offset=0):
        kind = F.BM_BUF_AXON_STATES if buf == "axon_states" else F.BUF[buf]
        li = 0 if kind == F.BM_BUF_AXON_STATES else self.data_layer(layer)
        a = np.ascontiguousarray(data)
        a = a.view(np.uint8) if a.dtype.itemsize == 1 else a.astype(np.uint8)
        F.check(self.lib.bm_area_write(self.h, kind, li, int(offset), a.ctypes.data_as(C.c_void_p), a.nbytes))

    def fill(self, buf, value, layer=0):
        n = int(self.plan.n_axons) if buf == "axon_states" else int(self.plan.layers[self.data_layer(layer)].buf_len[F.BUF[buf]])
        self.write(buf, np.full(n, value, dtype=np.int8 if buf in F.SIGNED_BUFS else np.uint8), layer)

    def read_slab(self):
        out = np.empty(self.slab_bytes, dtype=np.uint8)
        F.check(self.lib.bm_area_read_slab(self.h, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def write_slab(self, data):
        a = np.ascontiguousarray(data, dtype=np.uint8)
        F.check(self.lib.bm_area_write_slab(self.h, a.ctypes.data_as(C.c_void_p), a.nbytes))

    def cycle_count(self):
        v = C.c_uint64()
        F.check(self.lib.bm_area_get_cycle(self.h, C.byref(v)))
        return v.value

    def set_cycle(self, c):
        F.check(self.lib.bm_area_set_cycle(self.h, C.c_uint64(c)))

    def device_errors(self):
        """The area's sticky device error bits (bit 0: a bounded wait gave up)."""
        v = C.c_uint32()
        rc = self.lib.bm_area_device_errors(self.h, C.byref(v))
        if rc not in (F.BM_OK, F.BM_ERR_TIMEOUT):
            F.check(rc)
        return v.value

    def clear_errors(self):
        F.check(self.lib.bm_area_clear_errors(self.h))

    def set_wait_limit(self, us):
        """Limit of each bounded wait in the tuft kernels, microseconds (0: default)."""
        F.check(self.lib.bm_area_set_wait_limit(self.h, int(us)))

    def inject_stall(self, stage):
        """Fault injection: in each tiled tuft launch, the block that takes
        the tuft's first tile withholds the `stage`-th stage it issues from
        that tile on (from 1; 0: off)."""
        F.check(self.lib.bm_area_inject_stall(self.h, int(stage)))

    def tuft_form(self, layer, tuft):
        """How the fused path runs a tuft (bm_area_tuft_form): a dict of the
        bm_tuft_form fields."""
        f = F.bm_tuft_form()
        F.check(self.lib.bm_area_tuft_form(self.h, self.data_layer(layer), int(tuft), C.byref(f)))
        return {n: int(getattr(f, n)) for n, _ in F.bm_tuft_form._fields_}

    def slab_ptr(self):
        p = C.c_void_p()
        F.check(self.lib.bm_area_slab_ptr(self.h, C.byref(p)))
        return p.value

    def deliver_tract(self, src, src_output, dst_input, dst_offset):
        """bm_area_deliver_tract: src's current output `src_output` into this
        area's input `dst_input` at axon `dst_offset`, on this area's stream."""
        F.check(self.lib.bm_area_deliver_tract(src.h, int(src_output), self.h, int(dst_input),
                                               C.c_uint64(int(dst_offset))))

    def axons_touched(self):
        """Orders the next cycle's front steps after axon reads or writes the
        caller queued on the area's stream through slab_ptr
        (bm_area_axons_touched)."""
        F.check(self.lib.bm_area_axons_touched(self.h))

    def side_steps(self):
        """Steps of the cycle that run beside the chain of dependent steps."""
        v = C.c_uint32()
        F.check(self.lib.bm_area_side_steps(self.h, C.byref(v)))
        return v.value

    def front_steps(self):
        """Leading steps of the cycle that run on the front stream, beside the
        previous cycle's later steps (0: none this cycle)."""
        v = C.c_uint32()
        F.check(self.lib.bm_area_front_steps(self.h, C.byref(v)))
        return v.value

    def sampler(self, kind, layer=None, backpressure=False):
        """CorticalArea::sampler: a Sampler over `kind` (a SAMPLER_KINDS name)
        of data layer `layer` (name or index; for "axons", None = every axon)."""
        return Sampler(self, kind, layer, backpressure)

    # ---- timing ----
    def set_profiling(self, on):
        F.check(self.lib.bm_area_set_profiling(self.h, 1 if on else 0))

    def profile(self):
        n = 32
        names = (C.c_char_p * n)()
        launches = (C.c_uint64 * n)()
        ms = (C.c_double * n)()
        got = C.c_uint32()
        F.check(self.lib.bm_area_get_profile(self.h, n, names, launches, ms, C.byref(got)))
        return {names[i].decode(): (int(launches[i]), float(ms[i])) for i in range(got.value)}

    def reset_profile(self):
        F.check(self.lib.bm_area_reset_profile(self.h))

    def launches_per_cycle(self):
        v = C.c_uint32()
        F.check(self.lib.bm_area_launches_per_cycle(self.h, C.byref(v)))
        return v.value

    def close(self):
        if self.h:
            # A batch that holds this area goes first (it points into the area).
            for r in getattr(self, "_holders", []):
                b = r()
                if b is not None:
                    b.close()
            self._holders = []
            # The library destroys the area's samplers with it.
            for r in self._samplers:
                smp = r()
                if smp is not None:
                    smp.h = C.c_void_p()
            self._samplers = []
            self.lib.bm_area_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# Sampler kinds (SamplerKind, src/cortex/cortical_area.rs:61-90) -> buffer kind.
SAMPLER_KINDS = {
    "axons": F.BM_BUF_AXON_STATES,
    "soma_states": F.BUF["cel_states"], "soma_energies": F.BUF["cel_energies"],
    "soma_activities": F.BUF["cel_activities"], "soma_flag_sets": F.BUF["cel_flag_sets"],
    "tuft_states": F.BUF["tft_states"], "tuft_best_den_ids": F.BUF["tft_best_den_ids"],
    "tuft_best_den_states_raw": F.BUF["tft_best_den_states_raw"],
    "tuft_best_den_states": F.BUF["tft_best_den_states"], "tuft_prev_states": F.BUF["tft_prev_states"],
    "tuft_prev_best_den_ids": F.BUF["tft_prev_best_den_ids"],
    "tuft_prev_best_den_states_raw": F.BUF["tft_prev_best_den_states_raw"],
    "tuft_prev_best_den_states": F.BUF["tft_prev_best_den_states"],
    "den_states": F.BUF["den_states"], "den_states_raw": F.BUF["den_states_raw"],
    "den_energies": F.BUF["den_energies"], "den_activities": F.BUF["den_activities"],
    "den_thresholds": F.BUF["den_thresholds"],
    "syn_states": F.BUF["syn_states"], "syn_strengths": F.BUF["syn_strengths"],
    "syn_src_slc_ids": F.BUF["syn_src_slc_ids"], "syn_src_col_v_offs": F.BUF["syn_src_col_v_offs"],
    "syn_src_col_u_offs": F.BUF["syn_src_col_u_offs"], "syn_flag_sets": F.BUF["syn_flag_sets"],
}
SIGNED_KINDS = {"syn_strengths", "syn_src_col_v_offs", "syn_src_col_u_offs"}


class Sampler:
    """Per-cycle readback of one buffer of an area (CorticalArea::sampler,
    src/cortex/cortical_area.rs:1017-1284) through a one-frame channel with
    the tract channel's send / skip / backpressure rules
    (src/subcortex/tract_channel.rs:400-488); bm_sampler_* in
    include/bismit_b200.h."""

    def __init__(self, area, kind, layer=None, backpressure=False):
        self.lib = F.lib()
        self.area = area
        self.kind = kind
        buf = SAMPLER_KINDS[kind]
        if layer is None:
            if kind != "axons":
                raise ValueError("sampler %r needs a layer" % kind)
            li = F.BM_ALL_LAYERS
        else:
            li = area.data_layer(layer) if isinstance(layer, str) else int(layer)
        self.h = C.c_void_p()
        F.check(self.lib.bm_sampler_create(area.h, buf, li, 1 if backpressure else 0, C.byref(self.h)))
        n = C.c_uint64()
        F.check(self.lib.bm_sampler_len(self.h, C.byref(n)))
        self.len = n.value
        area._samplers.append(weakref.ref(self))

    def recv(self, wait_for_frame=False):
        """(cycle, frame) of the unread frame, or None (TractReceiver::recv)."""
        out = np.empty(self.len, np.uint8)
        cyc = C.c_uint64()
        got = C.c_int()
        F.check(self.lib.bm_sampler_recv(self.h, 1 if wait_for_frame else 0, out.ctypes.data, self.len,
                                         C.byref(cyc), C.byref(got)))
        if not got.value:
            return None
        return cyc.value, (out.view(np.int8) if self.kind in SIGNED_KINDS else out)

    def set_backpressure(self, on):
        prior = C.c_int()
        F.check(self.lib.bm_sampler_set_backpressure(self.h, 1 if on else 0, C.byref(prior)))
        return bool(prior.value)

    def set_timeout(self, ms):
        F.check(self.lib.bm_sampler_set_timeout(self.h, int(ms)))

    def stats(self):
        sent, skipped = C.c_uint64(), C.c_uint64()
        F.check(self.lib.bm_sampler_stats(self.h, C.byref(sent), C.byref(skipped)))
        return {"sent": sent.value, "skipped": skipped.value}

    def close(self):
        if self.h and self.area.h:
            self.lib.bm_sampler_destroy(self.h)
        self.h = C.c_void_p()


class Batch:
    """Areas of one layer map (uneven sizes allowed) cycled together: one
    launch per stage step for all of them, the cycle replayed from a CUDA
    graph (bm_batch_*, include/bismit_b200.h). Each area's bytes after a
    batched cycle equal its bytes after cycling it alone."""

    def __init__(self, ctx, areas, graph=True):
        self.lib = F.lib()
        self.ctx = ctx
        self.areas = list(areas)
        hs = (C.c_void_p * len(self.areas))(*[a.h.value for a in self.areas])
        self.h = C.c_void_p()
        F.check(self.lib.bm_batch_create(ctx.h, hs, len(self.areas), C.byref(self.h)))
        ctx._adopt(self)
        for a in self.areas:
            a._holders.append(weakref.ref(self))
        if not graph:
            self.set_graph(False)

    def set_graph(self, on):
        F.check(self.lib.bm_batch_set_graph(self.h, 1 if on else 0))

    def cycle(self, n=1):
        F.check(self.lib.bm_batch_cycle(self.h, int(n)))

    def frame_bytes(self):
        v = C.c_uint64()
        F.check(self.lib.bm_batch_frame_bytes(self.h, C.byref(v)))
        return v.value

    def cycle_frames_device(self, dev_ptr, n):
        """n cycles; cycle k first takes its frame block (input 0 of every area,
        packed in batch order) from dev_ptr + k * frame_bytes()."""
        F.check(self.lib.bm_batch_cycle_frames_device(self.h, C.c_void_p(dev_ptr), int(n)))

    def pack_frames(self, per_area_frames):
        """Host-side packing: per_area_frames[a] is an (n, len_a) array; returns
        the (n, frame_bytes) array cycle_frames_device expects."""
        return np.ascontiguousarray(np.concatenate([np.asarray(f, np.uint8) for f in per_area_frames], axis=1))

    def launches_per_cycle(self):
        v = C.c_uint32()
        F.check(self.lib.bm_batch_launches_per_cycle(self.h, C.byref(v)))
        return v.value

    def device_errors(self):
        v = C.c_uint32()
        rc = self.lib.bm_batch_device_errors(self.h, C.byref(v))
        if rc not in (F.BM_OK, F.BM_ERR_TIMEOUT):
            F.check(rc)
        return v.value

    STEP_NAMES = {0: "tuft", 1: "tufts_plain", 2: "ssc_cycle", 3: "inhib_simple", 4: "inhib_passthrough",
                  5: "pyr_output", 6: "inhib_intra_column", 7: "pyr_cycle", 8: "tft_dst_mtp", 9: "ssc_mtp_simple",
                  10: "cycle_end", 11: "inhib_mtp", 12: "pyr_tail", 13: "regrow", 14: "smooth_activity",
                  1000: "fused_tuft_batch"}

    def set_profiling(self, on):
        F.check(self.lib.bm_batch_set_profiling(self.h, 1 if on else 0))

    def profile(self):
        """[(step name, layer, index, areas, launches, device ms)] of the steps that ran."""
        n = 64
        arrs = [(C.c_uint32 * n)() for _ in range(4)]
        launches = (C.c_uint64 * n)()
        ms = (C.c_double * n)()
        got = C.c_uint32()
        F.check(self.lib.bm_batch_get_profile(self.h, n, *arrs, launches, ms, C.byref(got)))
        out = []
        for i in range(got.value):
            k = int(arrs[0][i])
            name = self.STEP_NAMES.get(k, self.STEP_NAMES[1000] if k >= 1000 else str(k))
            out.append((name, int(arrs[1][i]), int(arrs[2][i]), int(arrs[3][i]), int(launches[i]), float(ms[i])))
        return out

    def reset_profile(self):
        F.check(self.lib.bm_batch_reset_profile(self.h))

    def autotune(self, cache_path=None):
        n = C.c_uint32()
        F.check(self.lib.bm_batch_autotune(self.h, cache_path.encode() if cache_path else None, C.byref(n)))
        return n.value

    def close(self):
        if self.h:
            self.lib.bm_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching serving of cortex sessions (bm_server_*,
    include/bismit_b200.h): sessions are admitted by device-memory budget,
    stay resident, and every tick cycles all resident sessions that have a
    pending frame in one batch."""

    def __init__(self, ctx, budget_bytes=0):
        self.lib = F.lib()
        self.ctx = ctx
        self.h = C.c_void_p()
        F.check(self.lib.bm_server_create(ctx.h, C.c_uint64(int(budget_bytes)), C.byref(self.h)))
        ctx._adopt(self)

    def open(self, desc, seed):
        sid = C.c_uint32()
        F.check(self.lib.bm_server_open(self.h, C.byref(desc), C.c_uint64(seed), C.byref(sid)))
        return sid.value

    def submit(self, sid, frames):
        a = np.ascontiguousarray(frames, dtype=np.uint8)
        if a.ndim == 1:
            a = a[None, :]
        F.check(self.lib.bm_server_submit(self.h, sid, a.ctypes.data_as(C.c_void_p), a.shape[1], a.shape[0]))

    def cancel_session(self, sid):
        """Closes a session and discards its queued frames."""
        F.check(self.lib.bm_server_cancel(self.h, sid))

    def close_session(self, sid):
        F.check(self.lib.bm_server_close(self.h, sid))

    def tick(self):
        n = C.c_uint32()
        F.check(self.lib.bm_server_tick(self.h, C.byref(n)))
        return n.value

    def drain(self):
        """Completes every queued tick (ticks are pipelined two deep)."""
        F.check(self.lib.bm_server_drain(self.h))

    def read_output(self, sid, length):
        out = np.empty(int(length), np.uint8)
        done = C.c_uint64()
        F.check(self.lib.bm_server_read_output(self.h, sid, out.ctypes.data_as(C.c_void_p), out.nbytes,
                                               C.byref(done)))
        return out, done.value

    def session_slab(self, sid, slab_bytes):
        """The session's whole state (while resident)."""
        h = C.c_void_p()
        F.check(self.lib.bm_server_session_area(self.h, sid, C.byref(h)))
        if not h.value:
            return None
        out = np.empty(int(slab_bytes), np.uint8)
        F.check(self.lib.bm_area_read_slab(h, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def stats(self):
        st = F.bm_server_stats()
        F.check(self.lib.bm_server_get_stats(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in F.bm_server_stats._fields_}

    def reset_stats(self):
        F.check(self.lib.bm_server_reset_stats(self.h))

    def close(self):
        if self.h:
            self.lib.bm_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


PREVIOUS_CYCLE = "previous_cycle"
SAME_CYCLE = "same_cycle"


class Cortex:
    """A set of cortical areas (Cortex, src/cortex/cortex.rs:37-120). Outputs
    of one area that feed inputs of another (the thalamic routing of the area
    schemes) travel as tracts. Two timings:

    * PREVIOUS_CYCLE (the default): the areas are cycled together as one
      batch, one launch per stage step for all of them, and every tract
      carries its source's output of the previous cycle, copied at the head
      of each cycle.
    * SAME_CYCLE: bismit's own order. Cortex::cycle cycles the areas one after
      another in scheme order (src/cortex/cortex.rs:99-119), each starting
      with its intake (src/cortex/cortical_area.rs:716-719), so a tract from
      an earlier area carries that area's output of the same cycle and one
      from a later area its output of the previous cycle. Each area then runs
      its own launch sequence (slower than the batch).

    Inputs fed from outside (subcortical areas) are written per area with
    `area(name).write_input(..)`; `external_inputs()` lists them."""

    def __init__(self, lmaps, areas, settings=None, seed=0, device=0, ctx=None, tract_timing=PREVIOUS_CYCLE):
        if tract_timing not in (PREVIOUS_CYCLE, SAME_CYCLE):
            raise ValueError("tract_timing must be %r or %r" % (PREVIOUS_CYCLE, SAME_CYCLE))
        self._own_ctx = ctx is None
        self.ctx = _Ctx(device) if ctx is None else ctx
        self.tract_timing = tract_timing
        self.areas = {}
        self._order = []
        for a in areas.areas:
            if lmaps[a.layer_map_name].kind != LayerMapKind.Cortical:
                continue
            d = area_desc(a.name, lmaps, areas, settings)
            self.areas[a.name] = CorticalArea(self.ctx, d, seed, a.name)
            self._order.append(a.name)
        plans = [self.areas[n].plan for n in self._order]
        self.tracts, self.external = area_tracts(lmaps, areas, self._order, plans)
        self.batch = None
        if self._order and tract_timing == PREVIOUS_CYCLE:
            self.batch = Batch(self.ctx, [self.areas[n] for n in self._order])
            for (sk, so, dk, di, off, _n) in self.tracts:
                F.check(self.batch.lib.bm_batch_connect(self.batch.h, sk, so, dk, di, C.c_uint64(off)))

    @staticmethod
    def builder(lmaps, areas):
        return CortexBuilder(lmaps, areas)

    def cycle(self, n=1):
        """Cortex::cycle: every area once (src/cortex/cortex.rs:99-119)."""
        if self.batch is not None:
            self.batch.cycle(n)
            return
        areas = [self.areas[name] for name in self._order]
        for _ in range(n):
            for k, a in enumerate(areas):
                for (sk, so, dk, di, off, _n) in self.tracts:
                    if dk == k:
                        a.deliver_tract(areas[sk], so, di, off)
                a.cycle(1)

    def area(self, name):
        return self.areas[name]

    def area_names(self):
        return list(self._order)

    def external_inputs(self):
        """[(area name, input index, axon offset, axons, source area, source layer)]
        of the inputs no area of this cortex feeds."""
        return [(self._order[k], i, off, n, src, sl) for (k, i, off, n, src, sl) in self.external]

    def synchronize(self):
        self.ctx.synchronize()

    def close(self):
        if self.batch is not None:
            self.batch.close()
        for a in self.areas.values():
            a.close()
        if self._own_ctx:
            self.ctx.close()


class CortexBuilder:
    """Cortex::builder(..).ca_settings(..).build() (src/cortex/cortex.rs:158-201)."""

    def __init__(self, lmaps, areas):
        if not isinstance(lmaps, LayerMapSchemeList) or not isinstance(areas, AreaSchemeList):
            raise TypeError("Cortex.builder takes a LayerMapSchemeList and an AreaSchemeList")
        self.lmaps, self.areas_ = lmaps, areas
        self._settings = None
        self._seed = 0
        self._device = 0
        self._timing = PREVIOUS_CYCLE

    def tract_timing(self, timing):
        """PREVIOUS_CYCLE (batched) or SAME_CYCLE (bismit's area order)."""
        self._timing = timing
        return self

    def ca_settings(self, s):
        self._settings = s
        return self

    def seed(self, seed):
        self._seed = int(seed)
        return self

    def device(self, d):
        self._device = int(d)
        return self

    def build(self):
        return Cortex(self.lmaps, self.areas_, self._settings, self._seed, self._device, tract_timing=self._timing)
