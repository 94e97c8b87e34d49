"""Input encoders (src/encode/): frames for an area's inputs written by the
library's device encoders (bm_encode_* in include/bismit_b200.h).

The reference's encoders are host objects that write one tract frame per
cycle. Here the state machines stay on the host (which image or value comes
next), while the frames are written by kernels into device memory: a single
frame for bm_area_write_input_device, or a block of per-cycle frames for
bm_area_cycle_frames_device / bm_batch_cycle_frames_device.

    IdxData           src/encode/idx_data.rs        idx file reader (u8 data)
    IdxStreamer       src/encode/idx_streamer.rs    images -> hex frames, cycles_per_frame, loop_frames
    encode_2d_image   src/encode/mod.rs:66-93
    encode_hex_mold_scaled, HexMoldTest   src/encode/write/mod.rs:190-217, src/encode/hex_mold_test.rs
    encode_scalar     src/encode/write/mod.rs:28-172
    ReversoScalarSequence                src/encode/reverso_scalar_sequence.rs
    ScalarGlyphWriter, ScalarSequence, VectorEncoder
                      src/encode/write/scalar_glyph_writer.rs, src/encode/scalar_sequence.rs,
                      src/encode/vector_encoder.rs
    ScalarSdrWriter, ScalarSdrGradiant    src/encode/write/scalar_sdr_writer.rs, src/encode/scalar_sdr_gradiant.rs
    GlyphBuckets, GlyphSequences          src/encode/glyph_buckets.rs, src/encode/glyph_sequences.rs

Random bytes and waypoint indices, entropy-seeded in the reference, come
from a seeded stream (`seed`).
"""
import ctypes as C
import os

import numpy as np

from . import _ffi as F


def _torch():
    import torch
    return torch


def _ptr(t):
    return C.c_void_p(t.data_ptr())


# -------------------------------------------------------------------- idx --

class IdxData:
    """IdxData::new (src/encode/idx_data.rs:20-94): an idx file of unsigned
    bytes. `dims` are the header's sizes (big-endian u32s after the magic
    number); `data` holds the items, the last dimension fastest."""

    def __init__(self, file_path):
        self.file_path = os.fspath(file_path)
        with open(self.file_path, "rb") as f:
            magic = f.read(4)
            if len(magic) != 4:
                raise ValueError("couldn't read '%s': file too short" % self.file_path)
            if magic[2] != 8:
                raise ValueError("IDX file: '%s' does not contain unsigned bytes." % self.file_path)
            n_dims = magic[3]
            head = f.read(4 * n_dims)
            if len(head) != 4 * n_dims:
                raise ValueError("couldn't read '%s': truncated header" % self.file_path)
            self.dims = [int.from_bytes(head[4 * i:4 * i + 4], "big") for i in range(n_dims)]
            n = int(np.prod(self.dims)) if self.dims else 0
            self.data = np.frombuffer(f.read(n), dtype=np.uint8)
            if self.data.size != n:
                raise ValueError("couldn't read '%s': %d of %d data bytes" % (self.file_path, self.data.size, n))

    @staticmethod
    def write(file_path, array):
        """Writes a uint8 array as an idx file (magic 0x00000803 for 3 dims)."""
        a = np.ascontiguousarray(array, dtype=np.uint8)
        with open(file_path, "wb") as f:
            f.write(bytes([0, 0, 8, a.ndim]))
            for d in a.shape:
                f.write(int(d).to_bytes(4, "big"))
            f.write(a.tobytes())


def encode_2d_image(ctx, images, src_dims, tar_dims, scale_factor, frames, frame_stride=None):
    """encode_2d_image over a batch: `images` (device, n x x_size x y_size
    bytes, rows of x_size), `src_dims` = (x_size, y_size), `tar_dims` =
    (v_size, u_size); frames (device) are `frame_stride` bytes apart (default
    v_size * u_size). Cells whose pixel lies outside the image keep their
    bytes."""
    x_size, y_size = src_dims
    v_size, u_size = tar_dims
    n = images.numel() // (x_size * y_size)
    stride = v_size * u_size if frame_stride is None else frame_stride
    F.check(F.lib().bm_encode_images(ctx.h, _ptr(images), n, x_size, y_size, C.c_float(scale_factor), _ptr(frames),
                                     stride, v_size, u_size))


class IdxStreamer:
    """IdxStreamer (src/encode/idx_streamer.rs): streams the images of a
    three-dimensional idx file (n x x_size x y_size) as hexagonal frames of
    `layer_dims` = (v_size, u_size), each image held for `cycles_per_frame`
    cycles; the images live in device memory once loaded."""

    def __init__(self, ctx, layer_dims, idx, cycles_per_frame, scale_factor):
        self.ctx = ctx
        self.layer_dims = tuple(layer_dims)
        self.idx_data = idx if isinstance(idx, IdxData) else IdxData(idx)
        dims = self.idx_data.dims
        if len(dims) > 3:
            raise ValueError("IdxStreamer::new(): Cannot handle idx files with more than three dimensions.")
        if len(dims) == 2:
            raise ValueError("One dimensional (linear) idx images not yet supported (trival to add).")
        if len(dims) != 3:
            raise ValueError("Idx files with more than three or less than one dimension(s) not supported.")
        self.image_dims = (dims[1], dims[2])
        if self.image_len() > self.layer_dims[0] * self.layer_dims[1]:
            raise ValueError("Ganglion vector size must be greater than or equal to IDX image size")
        self.cycles_per_frame = int(cycles_per_frame)
        self.scale_factor = float(scale_factor)
        self.repeat_counter = 0
        self.frame_counter = 0
        self.frames_count = dims[0]
        self._loop = None
        torch = _torch()
        self.images = torch.from_numpy(self.idx_data.data.copy()).to("cuda:%d" % ctx.device)

    def loop_frames(self, frames_to_loop):
        self._loop = int(frames_to_loop)
        return self

    def image_len(self):
        return self.image_dims[0] * self.image_dims[1]

    def increment_frame(self):
        """IdxStreamer::increment_frame (idx_streamer.rs:111-133)."""
        self.repeat_counter += 1
        if self.repeat_counter >= self.cycles_per_frame:
            self.repeat_counter = 0
            self.frame_counter += 1
            if self._loop is not None and self.frame_counter >= self._loop:
                self.frame_counter = 0
            if self.frame_counter >= self.frames_count:
                self.frame_counter = 0

    cycle_next = increment_frame

    def write_into(self, frame):
        """Encodes the current image into `frame` (device, v_size * u_size
        bytes), as InputGeneratorTract::write_into (idx_streamer.rs:166-193)."""
        n = self.image_len()
        img = self.images[self.frame_counter * n:(self.frame_counter + 1) * n]
        encode_2d_image(self.ctx, img, self.image_dims, self.layer_dims, self.scale_factor, frame)

    def frame_block(self, n_cycles, frames=None):
        """The next n_cycles frames (device, n_cycles x v_size * u_size), one
        per cycle, advancing the streamer as n_cycles cycles would. Frames of
        a block start from zeros, as the reference's tract buffer does."""
        torch = _torch()
        v, u = self.layer_dims
        if frames is None:
            frames = torch.zeros((n_cycles, v * u), dtype=torch.uint8, device=self.images.device)
        for c in range(n_cycles):
            self.write_into(frames[c])
            self.cycle_next()
        return frames


# --------------------------------------------------------------- hex mold --

def encode_hex_mold_scaled(ctx, radius, src_dims, tract_dims, frame):
    """A 1 at every offset of gen_syn_offs(radius, calc_scale(tract, src))
    around the frame's middle (`frame`: device, v_size * u_size bytes)."""
    v_size, u_size = tract_dims
    F.check(F.lib().bm_encode_hex_mold(ctx.h, int(radius), src_dims[0], src_dims[1], _ptr(frame), v_size, u_size))


class HexMoldTest:
    """HexMoldTest (src/encode/hex_mold_test.rs): the same hex mold every
    cycle."""

    def __init__(self, ctx, radius, src_dims, dst_dims):
        if radius < 0:
            raise ValueError("radius must be >= 0")
        torch = _torch()
        self.hex_mold = torch.zeros(dst_dims[0] * dst_dims[1], dtype=torch.uint8, device="cuda:%d" % ctx.device)
        encode_hex_mold_scaled(ctx, radius, src_dims, dst_dims, self.hex_mold)

    def write_into(self, frame):
        frame.copy_(self.hex_mold)

    def cycle_next(self):
        pass


# ----------------------------------------------------------------- scalars --

def encode_scalar(ctx, vals, val_range, tract_dims, frames, seed=0, frame_stride=None):
    """encode_scalar for each value (host floats) into frames (device)."""
    v_size, u_size = tract_dims
    a = np.ascontiguousarray(vals, dtype=np.float32)
    stride = v_size * u_size if frame_stride is None else frame_stride
    F.check(F.lib().bm_encode_scalar(ctx.h, a.ctypes.data_as(C.c_void_p), a.size, C.c_float(val_range[0]),
                                     C.c_float(val_range[1]), seed, _ptr(frames), stride, v_size, u_size))


class ScalarSdrWriter:
    """ScalarSdrWriter::new(val_range, way_span, tract_dims) and ::encode
    (src/encode/write/scalar_sdr_writer.rs:96-235)."""

    def __init__(self, ctx, val_range, way_span, tract_dims, seed=0):
        self.ctx = ctx
        self.val_range = (float(val_range[0]), float(val_range[1]))
        self.way_span = float(way_span)
        self.tract_dims = tuple(tract_dims)
        self.h = C.c_void_p()
        F.check(F.lib().bm_sdr_writer_create(ctx.h, C.c_float(self.val_range[0]), C.c_float(self.val_range[1]),
                                             C.c_float(self.way_span), tract_dims[0], tract_dims[1], seed,
                                             C.byref(self.h)))
        w, a, n = C.c_uint32(), C.c_uint32(), C.c_uint32()
        F.check(F.lib().bm_sdr_writer_info(self.h, C.byref(w), C.byref(a), C.byref(n)))
        self.way_count, self.sdr_active_count, self.sdr_len = w.value, a.value, n.value

    def waypoint_indices(self):
        out = np.zeros((self.way_count, self.sdr_active_count), np.uint32)
        F.check(F.lib().bm_sdr_writer_waypoints(self.h, out.ctypes.data_as(C.c_void_p), out.size))
        return out

    def encode(self, vals, frames, frame_stride=None):
        """One frame per value (host floats) into frames (device)."""
        a = np.atleast_1d(np.ascontiguousarray(vals, dtype=np.float32))
        stride = self.sdr_len if frame_stride is None else frame_stride
        F.check(F.lib().bm_sdr_writer_encode(self.h, a.ctypes.data_as(C.c_void_p), a.size, _ptr(frames), stride))

    def close(self):
        if self.h:
            F.lib().bm_sdr_writer_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ScalarSdrGradiant:
    """ScalarSdrGradiant (src/encode/scalar_sdr_gradiant.rs): a value stepping
    by `incr` through [lo, hi), wrapping to lo, written by a ScalarSdrWriter."""

    def __init__(self, ctx, val_range, way_span, incr, tract_dims, seed=0):
        self.range = (np.float32(val_range[0]), np.float32(val_range[1]))
        self.next = self.range[0]
        self.incr = np.float32(incr)
        self.writer = ScalarSdrWriter(ctx, val_range, way_span, tract_dims, seed)

    def increment_frame(self):
        self.next = np.float32(self.next + self.incr)   # f32 arithmetic, as for T = f32
        if self.next >= self.range[1]:
            self.next = self.range[0]

    cycle_next = increment_frame

    def write_into(self, frame):
        self.writer.encode([self.next], frame)


class ReversoScalarSequence:
    """ReversoScalarSequence (src/encode/reverso_scalar_sequence.rs): a value
    stepping by `incr` through [lo, hi), wrapping to lo; layer 0 gets
    encode_scalar(next), layer 1 encode_scalar(hi - next). Values are f32,
    as for T = f32."""

    def __init__(self, ctx, val_range, incr, tract_dims, seed=0):
        self.ctx = ctx
        self.range = (np.float32(val_range[0]), np.float32(val_range[1]))
        self.next = self.range[0]
        self.incr = np.float32(incr)
        self.tract_dims = tuple(tract_dims)
        self.seed = seed

    def increment_frame(self):
        self.next = np.float32(self.next + self.incr)
        if self.next >= self.range[1]:
            self.next = self.range[0]

    cycle_next = increment_frame

    def write_into(self, frame, layer):
        """Encodes into `frame` (device) for layer 0 or 1 (the reference
        panics on a third)."""
        if layer == 0:
            v = self.next
        elif layer == 1:
            v = np.float32(self.range[1] - self.next)
        else:
            raise ValueError("ReversoScalarSequence::write_into(): Too many layers!")
        encode_scalar(self.ctx, [v], (float(self.range[0]), float(self.range[1])), self.tract_dims, frame, self.seed)


def encode_scalar_glyph(ctx, vals, val_range, tract_dims, frames, frame_stride=None):
    """ScalarGlyphWriter::encode for each value (host floats) into frames
    (device), one frame per value."""
    v_size, u_size = tract_dims
    a = np.ascontiguousarray(vals, dtype=np.float32)
    stride = v_size * u_size if frame_stride is None else frame_stride
    F.check(F.lib().bm_encode_scalar_glyph(ctx.h, a.ctypes.data_as(C.c_void_p), a.size, C.c_float(val_range[0]),
                                           C.c_float(val_range[1]), _ptr(frames), stride, v_size, u_size))


class ScalarGlyphWriter:
    """ScalarGlyphWriter::new(val_range, tract_dims) and ::encode
    (src/encode/write/scalar_glyph_writer.rs:25-151)."""

    def __init__(self, ctx, val_range, tract_dims):
        if tract_dims[0] < 8 or tract_dims[1] < 8:
            raise ValueError("ScalarGlyphWriter::new(): Tract frame too small. Side lengths must each be "
                             "greater than 8.")
        if not val_range[0] <= val_range[1]:
            raise ValueError("ScalarGlyphWriter::new(): empty value range")
        self.ctx = ctx
        self.val_range = (float(val_range[0]), float(val_range[1]))
        self.tract_dims = tuple(tract_dims)

    def encode(self, vals, frames, frame_stride=None):
        encode_scalar_glyph(self.ctx, np.atleast_1d(vals), self.val_range, self.tract_dims, frames, frame_stride)


class ScalarSequence:
    """ScalarSequence (src/encode/scalar_sequence.rs): a value stepping by
    `incr` through [lo, hi), wrapping to lo, written by a ScalarGlyphWriter."""

    def __init__(self, ctx, val_range, incr, tract_dims):
        self.range = (np.float32(val_range[0]), np.float32(val_range[1]))
        self.next = self.range[0]
        self.incr = np.float32(incr)
        self.writer = ScalarGlyphWriter(ctx, val_range, tract_dims)

    def increment_frame(self):
        self.next = np.float32(self.next + self.incr)
        if self.next >= self.range[1]:
            self.next = self.range[0]

    cycle_next = increment_frame

    def write_into(self, frame):
        self.writer.encode([self.next], frame)


class VectorEncoder:
    """VectorEncoder (src/encode/vector_encoder.rs): one value per layer, each
    in its own range, each written by its layer's ScalarGlyphWriter.
    `values` is the external frame the caller fills (ext_frame_mut)."""

    def __init__(self, ctx, ranges, tract_dims):
        if len(ranges) != len(tract_dims):
            raise ValueError("VectorEncoder::new(): Range list length ('%d') and tract count ('%d') are not equal."
                             % (len(ranges), len(tract_dims)))
        self.ctx = ctx
        self.tract_dims = [tuple(t) for t in tract_dims]
        self.set_ranges(ranges)

    def set_ranges(self, ranges):
        """Resets the ranges and the number of scalars encoded (values to 0)."""
        if len(ranges) > len(self.tract_dims):
            raise ValueError("VectorEncoder::set_ranges(): Too many ranges provided ('%d'/'%d')."
                             % (len(ranges), len(self.tract_dims)))
        self.ranges = [tuple(r) for r in ranges]
        self.writers = [ScalarGlyphWriter(self.ctx, r, t) for r, t in zip(self.ranges, self.tract_dims)]
        self.values = np.zeros(len(self.ranges), np.float32)

    def write_into(self, frame, layer):
        """Layer `layer`'s value into `frame` (device); a layer past the
        ranges set writes nothing, as in the reference."""
        if layer >= len(self.tract_dims):
            raise ValueError("VectorEncoder::write_into(): No layer %d" % layer)
        if layer < len(self.writers):
            self.writers[layer].encode([self.values[layer]], frame)

    def cycle_next(self):
        pass


class GlyphBuckets:
    """GlyphBuckets (src/encode/glyph_buckets.rs): the images of an idx image
    file sorted into one bucket per label (10), and a cursor per bucket that
    cycles through its images."""

    BUCKET_COUNT = 10

    def __init__(self, label_file, image_file):
        labels = label_file if isinstance(label_file, IdxData) else IdxData(label_file)
        images = image_file if isinstance(image_file, IdxData) else IdxData(image_file)
        if len(images.dims) != 3:
            raise ValueError("GlyphBuckets::new(): Source idx file must have three dimensions.")
        if images.dims[0] != labels.dims[0]:
            raise ValueError("GlyphBuckets::new(): The images file must contain the same number of elements as "
                             "the labels file.")
        self.glyph_dims = (images.dims[1], images.dims[2])
        n = self.glyph_len()
        imgs = images.data.reshape(images.dims[0], n)
        lab = labels.data[:images.dims[0]]
        if lab.size and int(lab.max()) > self.BUCKET_COUNT:
            raise ValueError("GlyphBuckets::new(): label exceeds bucket count (%d)." % self.BUCKET_COUNT)
        # A label equal to the bucket count passes the reference's assert and
        # then indexes past its buckets.
        if lab.size and int(lab.max()) == self.BUCKET_COUNT:
            raise ValueError("GlyphBuckets::new(): label %d has no bucket" % self.BUCKET_COUNT)
        self.buckets = [imgs[lab == b].reshape(-1) for b in range(self.BUCKET_COUNT)]
        self.cursors = [0] * self.BUCKET_COUNT

    def glyph_len(self):
        return self.glyph_dims[0] * self.glyph_dims[1]

    def count(self):
        return len(self.buckets)

    def next_glyph(self, bucket_id):
        """The image under bucket_id's cursor; the cursor moves on (wrapping).
        An empty bucket is refused (the reference panics slicing it)."""
        if not 0 <= bucket_id < len(self.buckets):
            raise ValueError("GlyphBuckets::next_glyph(): bucket_id (%d) exceeds bucket count (%d)."
                             % (bucket_id, len(self.buckets)))
        b = self.buckets[bucket_id]
        if b.size == 0:
            raise ValueError("GlyphBuckets::next_glyph(): bucket %d holds no glyph" % bucket_id)
        z = self.cursors[bucket_id]
        g = b[z:z + self.glyph_len()]
        z += self.glyph_len()
        self.cursors[bucket_id] = 0 if z == b.size else z
        return g


class GlyphSequences:
    """GlyphSequences (src/encode/glyph_sequences.rs): `seq_count` sequences
    of bucket ids, lengths uniform in seq_lens (inclusive), drawn from a
    seeded stream (the reference's is entropy-seeded); a cursor walks them.
    The image layer gets the next glyph of the cursor's bucket through
    encode_2d_image; the value layer (dims 1 x hrz_dims) gets idx & 0xFF.
    Every write draws a glyph from the bucket, as the reference's write_into
    does for either layer."""

    def __init__(self, ctx, seq_lens, seq_count, scale, hrz_dims, img_layer_dims, label_file, image_file, seed=0):
        if seq_lens[1] < seq_lens[0]:
            raise ValueError("GlyphSequences::new(): Sequence length range ('seq_lens') invalid. High end must at "
                             "least be equal to low end: '%r'." % (tuple(seq_lens),))
        self.ctx = ctx
        self.buckets = GlyphBuckets(label_file, image_file)
        self.scale = float(scale)
        self.img_layer_dims = tuple(img_layer_dims)
        self.val_layer_dims = (int(hrz_dims[0]), int(hrz_dims[1]))
        rng = np.random.default_rng([int(seed) & 0xFFFFFFFF, 0x676C7970])
        self.sequences = []
        for _ in range(seq_count):
            n = int(rng.integers(seq_lens[0], seq_lens[1] + 1))
            self.sequences.append([int(x) for x in rng.integers(0, self.buckets.count(), n)])
        self.seq_idx = 0
        self.gly_idx = 0
        torch = _torch()
        self._device = torch.device("cuda:%d" % ctx.device)

    def get(self):
        return self.seq_idx, self.sequences[self.seq_idx][self.gly_idx]

    def advance(self):
        """SeqReader::advance (glyph_sequences.rs:28-36)."""
        self.gly_idx += 1
        if self.gly_idx >= len(self.sequences[self.seq_idx]):
            self.gly_idx = 0
            self.seq_idx += 1
            if self.seq_idx >= len(self.sequences):
                self.seq_idx = 0

    cycle_next = advance

    def write_into(self, frame, layer):
        """layer "img" or "val"; `frame` (device) of that layer's dims."""
        torch = _torch()
        _, glyph_id = self.get()
        glyph = self.buckets.next_glyph(glyph_id)
        if layer == "img":
            img = torch.from_numpy(np.ascontiguousarray(glyph)).to(self._device)
            encode_2d_image(self.ctx, img, self.buckets.glyph_dims, self.img_layer_dims, self.scale, frame)
        elif layer == "val":
            n = self.val_layer_dims[0] * self.val_layer_dims[1]
            frame[:n].copy_(torch.arange(n, device=self._device, dtype=torch.int64).bitwise_and(0xFF).to(torch.uint8))
        else:
            raise ValueError("GlyphSequences::write_into(): Layer address not found: %r." % (layer,))
