"""Input encoders (src/encode/): the oracle's C restatement checked on the
CPU (against a float32 numpy restatement of encode_2d_image, gen_syn_offs for
the hex mold, and the geometry of the border and SDR encoders), and the
device encoders (bm_encode_*) against the oracle byte for byte on the GPU."""
import ctypes as C

import numpy as np
import pytest

import oracle
from bismit_b200 import _ffi as F, configs, cortex, encode as E, map as M

f32 = np.float32


def _image_py(img, scale, v_size, u_size):
    """encode_2d_image (src/encode/mod.rs:36-93) in numpy float32 scalars,
    operation by operation; calc_offs receives (x_size, y_size) in the slots
    it names (y_size, x_size)."""
    y_size, x_size = img.shape

    def to_pixel(v, u, hs, xo, yo):
        u_inv = f32(0.0) - f32(u)
        w_inv = f32(v) + f32(u)
        x = w_inv * f32(1.5) * hs
        y = (u_inv + (w_inv / f32(2.0))) * f32(1.73205080756) * hs
        return x - xo, y + yo

    hs = f32(x_size + y_size) / (f32(scale) * f32(v_size + u_size))
    co_y, co_x = x_size, y_size
    xi, yi = to_pixel(v_size >> 1, u_size >> 1, hs, f32(0), f32(0))
    xo, yo = xi - f32(co_x >> 1), f32(co_y >> 1) - yi
    out = np.zeros(v_size * u_size, np.uint8)
    for v in range(v_size):
        for u in range(u_size):
            x, y = to_pixel(v, u, hs, xo, yo)
            if f32(0) <= y < f32(y_size) and f32(0) <= x < f32(x_size):
                out[v * u_size + u] = img.reshape(-1)[int(y) * x_size + int(x)]
    return out


def test_idx_data_round_trip_and_refusals(tmp_path):
    rng = np.random.default_rng(0)
    a = rng.integers(0, 256, size=(5, 28, 28), dtype=np.uint8)
    p = tmp_path / "imgs.idx"
    E.IdxData.write(p, a)
    d = E.IdxData(p)
    assert d.dims == [5, 28, 28] and np.array_equal(d.data, a.reshape(-1))
    raw = open(p, "rb").read()
    bad = tmp_path / "f32.idx"
    bad.write_bytes(raw[:2] + bytes([0x0D]) + raw[3:])
    with pytest.raises(ValueError, match="does not contain unsigned bytes"):
        E.IdxData(bad)
    short = tmp_path / "short.idx"
    short.write_bytes(raw[:-10])
    with pytest.raises(ValueError, match="data bytes"):
        E.IdxData(short)


@pytest.mark.parametrize("shape,dims,scale", [((28, 28), (32, 32), 1.0), ((28, 28), (40, 24), 1.3),
                                              ((12, 20), (24, 40), 0.7), ((9, 31), (16, 16), 2.5)])
def test_image_encoder_matches_float32_restatement(shape, dims, scale):
    rng = np.random.default_rng(sum(shape) + dims[0])
    img = rng.integers(1, 256, size=shape, dtype=np.uint8)
    got = oracle.encode_image(img, scale, *dims)
    assert np.array_equal(got, _image_py(img, scale, *dims))
    assert np.count_nonzero(got) > 0


@pytest.mark.parametrize("radius,src,dims", [(4, (32, 32), (32, 32)), (3, (16, 16), (32, 32)), (6, (64, 48), (32, 32))])
def test_hex_mold_is_gen_syn_offs_around_the_middle(radius, src, dims):
    mold, n = oracle.hex_mold(radius, src, *dims)
    vs = (dims[0] * 1024) // max(1, (src[0] * 1024) // 16)
    us = (dims[1] * 1024) // max(1, (src[1] * 1024) // 16)
    ov, ou = oracle.gen_syn_offs(radius, vs, us)
    want = np.zeros(dims[0] * dims[1], np.uint8)
    for a, b in zip(ov.tolist(), ou.tolist()):
        want[(a + dims[0] // 2) * dims[1] + b + dims[1] // 2] = 1
    assert n == len(ov) and np.array_equal(mold, want)
    with pytest.raises(ValueError):
        oracle.hex_mold(40, (32, 32), 32, 32)      # leaves the frame


def test_scalar_encoder_draws_one_hexagon_along_the_border():
    v = u = 48
    r = (v + u) // 32
    vals = np.linspace(0, 100, 41, dtype=np.float32)
    frames = oracle.encode_scalar(vals, 0.0, 100.0, 9, v, u)
    centers = []
    for fr in frames:
        nz = np.nonzero(fr)[0]
        assert len(nz) == 3 * r * r + 3 * r + 1
        assert fr[nz].min() >= 64 and fr[nz].max() <= 127
        rows, cols = nz // u, nz % u
        centers.append((int(round(rows.mean())), int(round(cols.mean()))))
    margin = 2 * r + 2
    for cv, cu in centers:
        assert cv in (margin, v - margin - 1) or cu in (margin, u - margin - 1)
    assert centers[0] == centers[-1]                     # the top of the range wraps to the start
    assert len(set(centers)) > 30
    with pytest.raises(ValueError):
        oracle.encode_scalar([100.5], 0.0, 100.0, 9, v, u)


def test_sdr_writer_waypoints_blend():
    v = u = 32
    ways = oracle.sdr_waypoints(0.0, 10.0, 3.0, v, u, 5)
    active = v * u // 48
    assert ways.shape == (int(np.ceil(10 / 3)) + 1, active) and ways.max() < v * u
    frames = oracle.sdr_encode([0.0, 3.0, 4.5, 10.0], 0.0, 10.0, 3.0, ways, v * u)
    for k, val in enumerate([0.0, 3.0]):            # on a waypoint: that waypoint's SDR
        want = np.zeros(v * u, np.uint8)
        want[ways[k]] = 128
        assert np.array_equal(frames[k], want)
    mid = np.zeros(v * u, np.uint8)                   # halfway: half of each, way 1 from its start
    mid[ways[1][:active - active // 2]] = 128
    mid[ways[2][:active // 2]] = 128
    assert np.array_equal(frames[2], mid)
    with pytest.raises(ValueError):                   # the reference indexes past the last waypoint here
        oracle.sdr_encode([9.0], 0.0, 9.0, 3.0, oracle.sdr_waypoints(0.0, 9.0, 3.0, v, u, 5), v * u)


# ----------------------------------------------------------------- device --

@pytest.fixture(scope="module")
def ctx():
    c = cortex._Ctx(0)
    yield c
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("shape,dims,scale", [((28, 28), (32, 32), 1.0), ((12, 20), (24, 40), 0.7),
                                              ((9, 31), (16, 16), 2.5), ((28, 28), (128, 128), 1.0)])
def test_device_image_encoder_matches_oracle(ctx, shape, dims, scale):
    import torch
    rng = np.random.default_rng(7)
    n = 5
    imgs = rng.integers(0, 256, size=(n,) + shape, dtype=np.uint8)
    pre = rng.integers(0, 256, size=(n, dims[0] * dims[1] + 16), dtype=np.uint8)   # stride > frame
    dev_frames = torch.from_numpy(pre.copy()).cuda()
    E.encode_2d_image(ctx, torch.from_numpy(imgs).cuda(), (shape[1], shape[0]), dims, scale, dev_frames,
                      frame_stride=pre.shape[1])
    got = dev_frames.cpu().numpy()
    for k in range(n):
        want = oracle.encode_image(imgs[k], scale, *dims, target=pre[k, :dims[0] * dims[1]])
        assert np.array_equal(got[k, :dims[0] * dims[1]], want), k
        assert np.array_equal(got[k, dims[0] * dims[1]:], pre[k, dims[0] * dims[1]:])


@pytest.mark.gpu
def test_device_hex_mold_scalar_and_sdr_match_oracle(ctx):
    import torch
    mold = torch.zeros(32 * 32, dtype=torch.uint8, device="cuda")
    E.encode_hex_mold_scaled(ctx, 5, (24, 40), (32, 32), mold)
    assert np.array_equal(mold.cpu().numpy(), oracle.hex_mold(5, (24, 40), 32, 32)[0])
    with pytest.raises(F.BismitError):
        E.encode_hex_mold_scaled(ctx, 40, (32, 32), (32, 32), mold)

    vals = np.linspace(-5, 37, 29, dtype=np.float32)
    frames = torch.full((len(vals), 40 * 56), 7, dtype=torch.uint8, device="cuda")
    E.encode_scalar(ctx, vals, (-5.0, 37.0), (40, 56), frames, seed=11)
    assert np.array_equal(frames.cpu().numpy(), oracle.encode_scalar(vals, -5.0, 37.0, 11, 40, 56))
    with pytest.raises(F.BismitError):
        E.encode_scalar(ctx, [38.0], (-5.0, 37.0), (40, 56), frames)

    w = E.ScalarSdrWriter(ctx, (0.0, 20.0), 2.5, (48, 48), seed=3)
    ways = oracle.sdr_waypoints(0.0, 20.0, 2.5, 48, 48, 3)
    assert np.array_equal(w.waypoint_indices(), ways)
    vals = np.linspace(0, 19.9, 57, dtype=np.float32)
    frames = torch.full((len(vals), 48 * 48), 9, dtype=torch.uint8, device="cuda")
    w.encode(vals, frames)
    assert np.array_equal(frames.cpu().numpy(), oracle.sdr_encode(vals, 0.0, 20.0, 2.5, ways, 48 * 48))
    with pytest.raises(F.BismitError):
        w.encode([20.0], frames)          # 20 / 2.5 = waypoint 8, whose successor does not exist
    w.close()


@pytest.mark.gpu
def test_idx_streamer_feeds_an_area(ctx, tmp_path):
    """Images from an idx file, each held two cycles, streamed as a device
    frame block into bm_area_cycle_frames_device, against the oracle fed the
    oracle's own encoding of the same images."""
    import torch
    rng = np.random.default_rng(1)
    imgs = np.where(rng.random((3, 28, 28)) < 0.1, rng.integers(1, 256, (3, 28, 28)), 0).astype(np.uint8)
    p = tmp_path / "seq.idx"
    E.IdxData.write(p, imgs)
    area = cortex.CorticalArea(ctx, M.area_desc("v1", *configs.instance_area(32, 1, 8, 16), configs.bench_settings()), 4)
    plan = area.plan
    assert plan.inputs[0].len == 32 * 32
    slab = area.read_slab()
    s = E.IdxStreamer(ctx, (32, 32), p, cycles_per_frame=2, scale_factor=1.0).loop_frames(2)
    n = 6
    block = s.frame_block(n)
    torch.cuda.synchronize()
    area.cycle_frames_device(block.data_ptr(), 32 * 32, n)
    order = [0, 0, 1, 1, 0, 0]       # two images looped, two cycles each
    want = np.stack([oracle.encode_image(imgs[i], 1.0, 32, 32) for i in order])
    assert np.array_equal(block.cpu().numpy(), want)
    oracle.run(plan, slab, want, n, start_cycle=0)
    got = area.read_slab()
    assert np.array_equal(got, slab)
    area.close()


def _glyph_py(val, lo, hi, v_size, u_size):
    """ScalarGlyphWriter::new + ::encode (src/encode/write/scalar_glyph_
    writer.rs:25-151) in numpy float32 scalars, loop by loop."""
    radius = (v_size + u_size) // 32
    margin = radius + (radius + 1) + 1
    ttv, ttu = v_size - margin * 2 - 1, u_size - margin * 2 - 1
    total = ttv * 2 + ttu * 2
    sides = (ttu, ttu + ttv, 2 * ttu + ttv, total)
    pct = (f32(val) - f32(lo)) / (f32(hi) - f32(lo))
    t = np.floor(pct * f32(total))
    tile = 0 if not t > 0 else int(t)
    if tile < sides[0]:
        c = (margin, margin + tile)
    elif tile < sides[1]:
        c = (margin + (tile - sides[0]), margin + ttu)
    elif tile < sides[2]:
        c = (margin + ttv, (margin + ttu) - (tile - sides[1]))
    elif tile < sides[3]:
        c = ((margin + ttv) - (tile - sides[2]), margin)
    else:
        assert tile == total
        c = (margin, margin)
    out = np.zeros(v_size * u_size, np.uint8)
    for v in range(-radius, radius + 1):
        for u in range(max(-radius, -v - radius), min(radius, -v + radius) + 1):
            out[(v + c[0]) * u_size + u + c[1]] = 127
    return out


@pytest.mark.parametrize("dims", [(32, 32), (48, 64), (8, 8), (96, 40)])
def test_scalar_glyph_writer_matches_loop_restatement(dims):
    """The oracle's C restatement of the glyph writer against a loop-by-loop
    float32 one, across the range's ends and every side of the track; values
    outside the range are refused."""
    lo, hi = -3.0, 7.5
    vals = np.concatenate([np.linspace(lo, hi, 57, dtype=np.float32), np.float32([hi, lo, 0.1])])
    got = oracle.encode_scalar_glyph(vals, lo, hi, *dims)
    for k, v in enumerate(vals):
        assert np.array_equal(got[k], _glyph_py(v, lo, hi, *dims)), (dims, float(v))
    r = (dims[0] + dims[1]) // 32
    assert all(np.count_nonzero(g) == 3 * r * r + 3 * r + 1 for g in got)
    with pytest.raises(ValueError):
        oracle.encode_scalar_glyph([np.float32(hi + 1)], lo, hi, *dims)


def test_glyph_buckets_and_sequences_cycle(tmp_path):
    """GlyphBuckets sorts images by label and cycles each bucket; GlyphSequences'
    sequences have lengths in range and ids below the bucket count, and its
    cursor walks them in order (src/encode/glyph_buckets.rs,
    src/encode/glyph_sequences.rs:13-36)."""
    rng = np.random.default_rng(1)
    n = 40
    labels = rng.integers(0, 10, n, dtype=np.uint8)
    images = rng.integers(0, 256, (n, 6, 5), dtype=np.uint8)
    E.IdxData.write(tmp_path / "labels.idx", labels)
    E.IdxData.write(tmp_path / "images.idx", images)
    b = E.GlyphBuckets(tmp_path / "labels.idx", tmp_path / "images.idx")
    assert b.glyph_dims == (6, 5) and b.count() == 10
    lab = int(labels[0])
    members = [images[i].reshape(-1) for i in range(n) if labels[i] == lab]
    for k in range(2 * len(members) + 1):
        assert np.array_equal(b.next_glyph(lab), members[k % len(members)])
    with pytest.raises(ValueError):
        b.next_glyph(10)


@pytest.mark.gpu
def test_device_glyph_and_sequence_encoders_match_oracle(ctx, tmp_path):
    """The device glyph writer and the sequence / vector encoders built on it
    against the oracle, frame for frame; GlyphSequences' image frames against
    the oracle's encode_2d_image of the glyph its cursor picks."""
    import torch
    dims = (48, 64)
    lo, hi = 0.0, 10.0
    vals = np.linspace(lo, hi, 41, dtype=np.float32)
    fr = torch.zeros((len(vals), dims[0] * dims[1]), dtype=torch.uint8, device="cuda:0")
    E.encode_scalar_glyph(ctx, vals, (lo, hi), dims, fr)
    assert np.array_equal(fr.cpu().numpy(), oracle.encode_scalar_glyph(vals, lo, hi, *dims))
    # ScalarSequence: f32 steps wrapping at hi.
    seq = E.ScalarSequence(ctx, (lo, hi), 0.7, dims)
    expect = []
    one = torch.zeros(dims[0] * dims[1], dtype=torch.uint8, device="cuda:0")
    for _ in range(20):
        seq.write_into(one)
        expect.append(seq.next)
        assert np.array_equal(one.cpu().numpy(), oracle.encode_scalar_glyph([seq.next], lo, hi, *dims)[0])
        seq.cycle_next()
    assert min(expect) == np.float32(lo) and max(expect) < np.float32(hi)
    # VectorEncoder: one value per layer, each in its range.
    ve = E.VectorEncoder(ctx, [(0.0, 1.0), (-5.0, 5.0)], [dims, (32, 32)])
    ve.values[:] = [0.25, -4.0]
    out0 = torch.zeros(dims[0] * dims[1], dtype=torch.uint8, device="cuda:0")
    out1 = torch.zeros(32 * 32, dtype=torch.uint8, device="cuda:0")
    ve.write_into(out0, 0)
    ve.write_into(out1, 1)
    assert np.array_equal(out0.cpu().numpy(), oracle.encode_scalar_glyph([0.25], 0.0, 1.0, *dims)[0])
    assert np.array_equal(out1.cpu().numpy(), oracle.encode_scalar_glyph([-4.0], -5.0, 5.0, 32, 32)[0])
    # ReversoScalarSequence: encode_scalar(next) and encode_scalar(hi - next).
    rs = E.ReversoScalarSequence(ctx, (0.0, 8.0), 1.5, dims, seed=4)
    rs.cycle_next()
    rs.write_into(out0, 0)
    assert np.array_equal(out0.cpu().numpy(), oracle.encode_scalar([rs.next], 0.0, 8.0, 4, *dims)[0])
    rs.write_into(out0, 1)
    assert np.array_equal(out0.cpu().numpy(),
                          oracle.encode_scalar([np.float32(8.0) - rs.next], 0.0, 8.0, 4, *dims)[0])
    # GlyphSequences.
    rng = np.random.default_rng(2)
    labels = rng.integers(0, 10, 60, dtype=np.uint8)
    images = rng.integers(0, 256, (60, 12, 12), dtype=np.uint8)
    E.IdxData.write(tmp_path / "l.idx", labels)
    E.IdxData.write(tmp_path / "i.idx", images)
    gs = E.GlyphSequences(ctx, (2, 4), 5, 1.0, (8, 8), (32, 32), tmp_path / "l.idx", tmp_path / "i.idx", seed=3)
    assert all(2 <= len(q) <= 4 for q in gs.sequences)
    shadow = E.GlyphBuckets(tmp_path / "l.idx", tmp_path / "i.idx")
    img = torch.zeros(32 * 32, dtype=torch.uint8, device="cuda:0")
    for _ in range(12):
        _, gid = gs.get()
        glyph = shadow.next_glyph(gid)
        img.zero_()
        gs.write_into(img, "img")
        want = oracle.encode_image(glyph.reshape(12, 12), 1.0, 32, 32)
        assert np.array_equal(img.cpu().numpy(), want)
        gs.cycle_next()
