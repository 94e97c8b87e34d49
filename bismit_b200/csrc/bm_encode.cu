// bm_encode.cu -- input encoders writing tract frames in device memory.
//
// bismit's encoders (src/encode/) are host code that writes one frame at a
// time. Here each is a kernel over a batch of frames in HBM, so a dataset or
// a block of values resident on the device becomes a frame block for
// bm_area_cycle_frames_device / bm_batch_cycle_frames_device without a host
// round trip:
//   * encode_2d_image (src/encode/mod.rs:66-93): hexagonal resampling of
//     images (the IdxStreamer's encoder, src/encode/idx_streamer.rs:158-161);
//   * encode_hex_mold_scaled (src/encode/write/mod.rs:190-217);
//   * encode_scalar (src/encode/write/mod.rs:28-172): a hexagon placed along
//     the frame's border by the value;
//   * ScalarSdrWriter (src/encode/write/scalar_sdr_writer.rs:96-235):
//     waypoint SDRs blended by the value.
// The float arithmetic is the reference's f32 arithmetic, operation by
// operation, in round-to-nearest intrinsics (no contraction), so frames are
// bit-exact against a CPU restatement. The reference draws its random bytes
// and waypoint indices from an entropy-seeded generator; here they come from
// a seeded splitmix64 stream.
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "bm_area.h"
#include "bm_layout.h"

using namespace bm;

namespace {

constexpr uint32_t kMaxEncodeValues = 4096;   // values per scalar-encoder call (one parameter block)
constexpr uint8_t kSdrAxonValue = 128;         // write_rand_subset_linear, scalar_sdr_writer.rs:33-35
constexpr uint32_t kSdrSparsity = 48;          // SPARSITY, scalar_sdr_writer.rs:13

__host__ __device__ inline uint64_t splitmix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// ---------------------------------------------------------------- images --

// The (x, y) pixel offsets of encode_2d_image (calc_offs, src/encode/mod.rs:
// 36-48; its caller passes the image's x size where calc_offs names y, and
// the reverse, which matters only for images that are not square).
struct ImageGeo {
    float hex_side, x_ofs, y_ofs;
};

// coord_hex_to_pixel, src/encode/mod.rs:52-72, evaluated as written.
__host__ __device__ inline void hex_to_pixel(float v, float u, float hex_side, float x_ofs, float y_ofs, float& x,
                                             float& y) {
#ifdef __CUDA_ARCH__
    const float w_inv = __fadd_rn(v, u);
    x = __fmul_rn(__fmul_rn(w_inv, 1.5f), hex_side);
    y = __fmul_rn(__fmul_rn(__fadd_rn(__fsub_rn(0.0f, u), __fdiv_rn(w_inv, 2.0f)), 1.73205080756f), hex_side);
    x = __fsub_rn(x, x_ofs);
    y = __fadd_rn(y, y_ofs);
#else
    volatile float w_inv = v + u;
    volatile float t = w_inv * 1.5f;
    x = t * hex_side;
    volatile float h = w_inv / 2.0f;
    volatile float u_inv = 0.0f - u;
    volatile float a = u_inv + h;
    volatile float b = a * 1.73205080756f;
    y = b * hex_side;
    x = x - x_ofs;
    y = y + y_ofs;
#endif
}

ImageGeo image_geo(uint32_t x_size, uint32_t y_size, float scale_factor, uint32_t v_size, uint32_t u_size) {
    ImageGeo g;
    volatile float num = (float)(x_size + y_size);
    volatile float den = scale_factor * (float)(v_size + u_size);
    g.hex_side = num / den;
    // calc_offs(v_size, u_size, x_size, y_size, hex_side) with its parameters
    // named (v_size, u_size, y_size, x_size, ..).
    const uint32_t cy = x_size, cx = y_size;
    float xo, yo;
    hex_to_pixel((float)(v_size >> 1), (float)(u_size >> 1), g.hex_side, 0.0f, 0.0f, xo, yo);
    volatile float xm = (float)(cx >> 1), ym = (float)(cy >> 1);
    g.x_ofs = xo - xm;
    g.y_ofs = ym - yo;
    return g;
}

// One thread per (image, v, u): the hexagon's pixel, when it falls inside the
// image, is copied to the frame; other cells keep what the frame held.
__global__ void k_encode_images(const uint8_t* __restrict__ images, uint32_t n, uint32_t x_size, uint32_t y_size,
                                ImageGeo g, uint8_t* __restrict__ frames, uint64_t stride, uint32_t v_size,
                                uint32_t u_size) {
    const uint64_t cells = (uint64_t)v_size * u_size;
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells * n) return;
    const uint64_t img = i / cells;
    const uint32_t c = (uint32_t)(i - img * cells);
    const uint32_t v = c / u_size, u = c - v * u_size;
    float x, y;
    hex_to_pixel((float)v, (float)u, g.hex_side, g.x_ofs, g.y_ofs, x, y);
    if (!(y >= 0.0f && y < (float)y_size && x >= 0.0f && x < (float)x_size)) return;
    const uint64_t src = (uint64_t)(uint32_t)y * x_size + (uint32_t)x;
    frames[img * stride + c] = images[img * (uint64_t)x_size * y_size + src];
}

// ------------------------------------------------------------- hex mold --

// encode_hex_mold_scaled: a 1 at every offset of gen_syn_offs(radius,
// scales) around the frame's middle. One thread per v offset; the u range
// of each row is gen_syn_offs's (src/map/syn_src.rs:47-149).
__global__ void k_hex_mold(int v_rad, int u_rad, uint32_t v_scale, uint32_t u_scale, uint8_t* frame, uint32_t v_size,
                           uint32_t u_size) {
    const int vo = -v_rad + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (vo > v_rad) return;
    const int vinv = -vo;
    const int a = max(-v_rad, vinv - v_rad), b = min(v_rad, vinv + v_rad);
    const int uz = (a * ((int)u_scale << 3)) / ((int)v_scale << 3);
    const int un = (b * ((int)u_scale << 3)) / ((int)v_scale << 3) + 1;
    (void)u_rad;
    for (int uo = uz; uo < un; uo++) {
        const int row = vo + (int)(v_size / 2), col = uo + (int)(u_size / 2);
        frame[(uint32_t)(row * (int)u_size + col)] = 1;
    }
}

// ------------------------------------------------------- border scalar --

struct ScalarArgs {
    uint32_t n;
    float hi;
    uint64_t key;
    float vals[kMaxEncodeValues];
};

// The hexagon's center for value `val` (encode_scalar, src/encode/write/
// mod.rs:44-112).
__device__ inline void scalar_center(float val, float hi, int v_size, int u_size, int& cv, int& cu) {
    const int radius = (v_size + u_size) / 32;
    const int margin = radius + (radius + 1) + 1;
    const int track_v = v_size - margin * 2 - 1, track_u = u_size - margin * 2 - 1;
    const float quad_size = __fdiv_rn(hi, 4.0f);
    const float quadrant = floorf(__fdiv_rn(val, quad_size));
    const float pos = __fsub_rn(val, __fmul_rn(quad_size, quadrant));
    auto to_tract = [&](int len) { return (int)__fmul_rn(__fdiv_rn(pos, quad_size), (float)len); };
    if (quadrant < 1.0f || quadrant >= 4.0f) {
        cv = margin;
        cu = to_tract(track_u) + margin;
    } else if (quadrant < 2.0f) {
        cv = to_tract(track_v) + margin;
        cu = u_size - margin - 1;
    } else if (quadrant < 3.0f) {
        cv = v_size - margin - 1;
        cu = u_size - (to_tract(track_u) + margin) - 1;
    } else {
        cv = v_size - (to_tract(track_v) + margin) - 1;
        cu = margin;
    }
}

// Zeroes a frame of len bytes with the block's threads, 16 bytes a store
// where the frame starts on a 16-byte boundary.
__device__ __forceinline__ void clear_frame(uint8_t* frame, uint32_t len) {
    uint32_t head = 0;
    if (((uintptr_t)frame & 15) == 0) {
        const uint32_t n16 = len / 16;
        for (uint32_t i = threadIdx.x; i < n16; i += blockDim.x) ((uint4*)frame)[i] = make_uint4(0, 0, 0, 0);
        head = n16 * 16;
    }
    for (uint32_t i = head + threadIdx.x; i < len; i += blockDim.x) frame[i] = 0;
}

// One block per frame: the frame is cleared, then the hexagon of radius
// (v + u) / 32 around the value's center gets bytes in 64..127.
__global__ void k_encode_scalar(const __grid_constant__ ScalarArgs A, uint8_t* __restrict__ frames, uint64_t stride,
                                uint32_t v_size, uint32_t u_size) {
    const uint32_t f = blockIdx.x;
    uint8_t* frame = frames + f * stride;
    const uint32_t len = v_size * u_size;
    clear_frame(frame, len);
    __syncthreads();
    int cv, cu;
    scalar_center(A.vals[f], A.hi, (int)v_size, (int)u_size, cv, cu);
    const int r = ((int)v_size + (int)u_size) / 32;
    const int side = 2 * r + 1;
    for (int k = threadIdx.x; k < side * side; k += blockDim.x) {
        const int v = -r + k / side, u = -r + k % side;
        if (u < max(-r, -v - r) || u > min(r, -v + r)) continue;
        const int row = v + cv, col = u + cu;
        if (row < 0 || row >= (int)v_size || col < 0 || col >= (int)u_size) continue;
        const uint32_t idx = (uint32_t)(row * (int)u_size + col);
        frame[idx] = (uint8_t)(64 + (splitmix(A.key + (uint64_t)f * len + idx) >> 58));
    }
}

// ---------------------------------------------------------- scalar glyph --

struct GlyphArgs {
    uint32_t n;
    int32_t radius;
    uint16_t cv[kMaxEncodeValues], cu[kMaxEncodeValues];   // each frame's hexagon center
};

// One block per frame (ScalarGlyphWriter::encode, src/encode/write/
// scalar_glyph_writer.rs:69-151): the frame is cleared, then the hexagon of
// radius `radius` around the frame's center is set to 127.
__global__ void k_encode_glyph(const __grid_constant__ GlyphArgs A, uint8_t* __restrict__ frames, uint64_t stride,
                               uint32_t v_size, uint32_t u_size) {
    const uint32_t f = blockIdx.x;
    uint8_t* frame = frames + f * stride;
    const uint32_t len = v_size * u_size;
    clear_frame(frame, len);
    __syncthreads();
    const int r = A.radius, side = 2 * r + 1, cv = A.cv[f], cu = A.cu[f];
    for (int k = threadIdx.x; k < side * side; k += blockDim.x) {
        const int v = -r + k / side, u = -r + k % side;
        if (u < max(-r, -v - r) || u > min(r, -v + r)) continue;
        frame[(uint32_t)((v + cv) * (int)u_size + u + cu)] = 127;
    }
}

// ------------------------------------------------------------ SDR writer --

struct SdrArgs {
    uint32_t n;
    uint32_t way0[kMaxEncodeValues / 2];
    uint16_t w0[kMaxEncodeValues / 2], w1[kMaxEncodeValues / 2];
};

// One block per frame: clear, then way 0's first w0 indices and way 1's first
// w1 indices are set to 128 (write_rand_subset_linear; the order of the two
// writes does not matter, both write the same byte).
__global__ void k_encode_sdr(const __grid_constant__ SdrArgs A, const uint32_t* __restrict__ ways, uint32_t active,
                             uint8_t* __restrict__ frames, uint64_t stride, uint32_t len) {
    const uint32_t f = blockIdx.x;
    uint8_t* frame = frames + f * stride;
    clear_frame(frame, len);
    __syncthreads();
    const uint32_t* w0 = ways + (uint64_t)A.way0[f] * active;
    const uint32_t* w1 = w0 + active;
    for (uint32_t k = threadIdx.x; k < A.w0[f]; k += blockDim.x) frame[w0[k]] = kSdrAxonValue;
    for (uint32_t k = threadIdx.x; k < A.w1[f]; k += blockDim.x) frame[w1[k]] = kSdrAxonValue;
}

}  // namespace

struct bm_sdr_writer_s {
    bm_ctx ctx = nullptr;
    float lo = 0, hi = 0, way_span = 0;
    uint32_t len = 0, active = 0, way_count = 0;
    uint32_t* ways = nullptr;   // device, way_count x active axon indices
};

extern "C" {

int bm_encode_images(bm_ctx ctx, const uint8_t* images, uint32_t n, uint32_t x_size, uint32_t y_size,
                     float scale_factor, uint8_t* frames, uint64_t frame_stride, uint32_t v_size, uint32_t u_size) {
    if (!ctx || (n && (!images || !frames))) return set_err(BM_ERR_INVALID, "null argument");
    if (!x_size || !y_size || !v_size || !u_size) return set_err(BM_ERR_INVALID, "encode_images: zero dims");
    if (!(scale_factor > 0.0f) || !std::isfinite(scale_factor))
        return set_err(BM_ERR_INVALID, "encode_images: scale factor must be positive");
    if (frame_stride < (uint64_t)v_size * u_size)
        return set_err(BM_ERR_INVALID, "encode_images: frame stride %llu below the frame's %u bytes",
                       (unsigned long long)frame_stride, v_size * u_size);
    if (!n) return BM_OK;
    const uint64_t threads = (uint64_t)v_size * u_size * n;
    if (threads > (uint64_t)0x7FFFFFFF * 256) return set_err(BM_ERR_UNSUPPORTED, "encode_images: too many cells");
    DevGuard g(ctx->device);
    const ImageGeo geo = image_geo(x_size, y_size, scale_factor, v_size, u_size);
    k_encode_images<<<(unsigned)((threads + 255) / 256), 256, 0, ctx->stream()>>>(images, n, x_size, y_size, geo,
                                                                                  frames, frame_stride, v_size, u_size);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? BM_OK : cuda_err(e, "encode_images");
}

int bm_encode_hex_mold(bm_ctx ctx, int32_t radius, uint32_t src_v_size, uint32_t src_u_size, uint8_t* frame,
                       uint32_t v_size, uint32_t u_size) {
    if (!ctx || !frame) return set_err(BM_ERR_INVALID, "null argument");
    if (radius < 0 || radius > 127) return set_err(BM_ERR_INVALID, "hex mold: radius %d outside 0..127", radius);
    if (!src_v_size || !src_u_size || !v_size || !u_size) return set_err(BM_ERR_INVALID, "hex mold: zero dims");
    // calc_scale(dst, src) per dimension (src/encode/write/mod.rs:196-197).
    auto scale = [](uint32_t dst, uint32_t src) -> int64_t {
        const uint64_t s = (uint64_t)dst * 1024, t = (uint64_t)src * 1024;
        const uint64_t incr = t < 16 ? 1 : t / 16;
        const uint64_t k = s / incr;
        return (k == 0 || k > 255) ? -1 : (int64_t)k;
    };
    const int64_t vs = scale(v_size, src_v_size), us = scale(u_size, src_u_size);
    if (vs < 0 || us < 0) return set_err(BM_ERR_INVALID, "hex mold: frame and source dims are more than 16x apart");
    int rv, ru;
    if (!offset_extent(radius, (uint32_t)vs, (uint32_t)us, &rv, &ru))
        return set_err(BM_ERR_INVALID, "hex mold: offsets beyond i8");
    // The reference writes unchecked; a mold that leaves the frame is refused.
    const int64_t mv = v_size / 2, mu = u_size / 2;
    if (mv - rv < 0 || mv + rv >= v_size || mu - ru < 0 || mu + ru >= u_size)
        return set_err(BM_ERR_INVALID, "hex mold: radius %d reaches outside a %u x %u frame", radius, v_size, u_size);
    DevGuard g(ctx->device);
    const int v_rad = (radius * (int)vs) >> 4, u_rad = (radius * (int)us) >> 4;
    const unsigned rows = (unsigned)(2 * v_rad + 1);
    k_hex_mold<<<(rows + 127) / 128, 128, 0, ctx->stream()>>>(v_rad, u_rad, (uint32_t)vs, (uint32_t)us, frame, v_size,
                                                              u_size);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? BM_OK : cuda_err(e, "hex mold");
}

int bm_encode_scalar(bm_ctx ctx, const float* vals, uint32_t n, float lo, float hi, uint64_t seed, uint8_t* frames,
                     uint64_t frame_stride, uint32_t v_size, uint32_t u_size) {
    if (!ctx || (n && (!vals || !frames))) return set_err(BM_ERR_INVALID, "null argument");
    if (n > kMaxEncodeValues) return set_err(BM_ERR_INVALID, "encode_scalar: at most %u values per call", kMaxEncodeValues);
    if (v_size < 8 || u_size < 8)
        return set_err(BM_ERR_INVALID, "encode::encode_scalar(): Tract frame too small. Side lengths must each be greater than 8.");
    if (frame_stride < (uint64_t)v_size * u_size) return set_err(BM_ERR_INVALID, "encode_scalar: frame stride too small");
    if (!(hi > 0.0f)) return set_err(BM_ERR_INVALID, "encode_scalar: the range's upper bound must be positive");
    ScalarArgs* A = new (std::nothrow) ScalarArgs;
    if (!A) return set_err(BM_ERR_OOM, "host allocation failed");
    std::memset(A, 0, sizeof *A);
    for (uint32_t k = 0; k < n; k++) {
        if (!(vals[k] >= lo && vals[k] <= hi)) {
            delete A;
            return set_err(BM_ERR_INVALID, "Unable to encode scalar value: '%g'. The value is outside of the allowed range: (%g, %g).",
                           (double)vals[k], (double)lo, (double)hi);
        }
        A->vals[k] = vals[k];
    }
    A->n = n;
    A->hi = hi;
    A->key = splitmix(seed ^ 0x656E636F64657273ull);
    int rc = BM_OK;
    if (n) {
        DevGuard g(ctx->device);
        k_encode_scalar<<<n, 256, 0, ctx->stream()>>>(*A, frames, frame_stride, v_size, u_size);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_err(e, "encode_scalar");
    }
    delete A;
    return rc;
}

int bm_encode_scalar_glyph(bm_ctx ctx, const float* vals, uint32_t n, float lo, float hi, uint8_t* frames,
                           uint64_t frame_stride, uint32_t v_size, uint32_t u_size) {
    if (!ctx || (n && (!vals || !frames))) return set_err(BM_ERR_INVALID, "null argument");
    if (n > kMaxEncodeValues) return set_err(BM_ERR_INVALID, "scalar glyph: at most %u values per call", kMaxEncodeValues);
    if (v_size < 8 || u_size < 8 || v_size > 0xFFFF || u_size > 0xFFFF)
        return set_err(BM_ERR_INVALID,
                       "ScalarGlyphWriter::new(): Tract frame too small. Side lengths must each be greater than 8.");
    if (frame_stride < (uint64_t)v_size * u_size) return set_err(BM_ERR_INVALID, "scalar glyph: frame stride too small");
    if (!(lo <= hi)) return set_err(BM_ERR_INVALID, "ScalarGlyphWriter::new(): empty value range");
    // ScalarGlyphWriter::new (scalar_glyph_writer.rs:25-67).
    const uint32_t radius = (v_size + u_size) / 32;
    const uint32_t margin = radius + (radius + 1) + 1;
    const uint32_t ttv = v_size - margin * 2 - 1, ttu = u_size - margin * 2 - 1;
    const uint32_t total = ttv * 2 + ttu * 2;
    const uint32_t side0 = ttu, side1 = ttu + ttv, side2 = 2 * ttu + ttv, side3 = total;
    volatile float span = hi - lo;
    GlyphArgs* A = new (std::nothrow) GlyphArgs;
    if (!A) return set_err(BM_ERR_OOM, "host allocation failed");
    std::memset(A, 0, sizeof *A);
    A->n = n;
    A->radius = (int32_t)radius;
    for (uint32_t k = 0; k < n; k++) {
        const float val = vals[k];
        if (!(val >= lo && val <= hi)) {
            delete A;
            return set_err(BM_ERR_INVALID,
                           "Unable to encode scalar value: '%g'. The value is outside of the allowed range: '(%g, %g)'.",
                           (double)val, (double)lo, (double)hi);
        }
        // f32 arithmetic as the reference's; `as u32` saturates (NaN -> 0).
        volatile float d = val - lo;
        volatile float pct = d / span;
        volatile float t = pct * (float)total;
        const float fl = std::floor((float)t);
        const uint32_t tile = !(fl > 0.0f) ? 0u : fl >= 4294967295.0f ? 0xFFFFFFFFu : (uint32_t)fl;
        uint32_t cv, cu;
        if (tile < side0) { cv = margin; cu = margin + tile; }
        else if (tile < side1) { cv = margin + (tile - side0); cu = margin + ttu; }
        else if (tile < side2) { cv = margin + ttv; cu = (margin + ttu) - (tile - side1); }
        else if (tile < side3) { cv = (margin + ttv) - (tile - side2); cu = margin; }
        else if (tile == total) { cv = margin; cu = margin; }
        else {
            delete A;
            return set_err(BM_ERR_INVALID, "ScalarGlyphWriter::encode: value %g maps past the track", (double)val);
        }
        A->cv[k] = (uint16_t)cv;
        A->cu[k] = (uint16_t)cu;
    }
    int rc = BM_OK;
    if (n) {
        DevGuard g(ctx->device);
        k_encode_glyph<<<n, 256, 0, ctx->stream()>>>(*A, frames, frame_stride, v_size, u_size);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_err(e, "scalar glyph");
    }
    delete A;
    return rc;
}

int bm_sdr_writer_create(bm_ctx ctx, float lo, float hi, float way_span, uint32_t v_size, uint32_t u_size,
                         uint64_t seed, bm_sdr_writer* out) {
    if (!ctx || !out) return set_err(BM_ERR_INVALID, "null argument");
    *out = nullptr;
    if (v_size < 8 || u_size < 8)
        return set_err(BM_ERR_INVALID, "ScalarSdrWriter::new(): Tract frame too small. Side lengths must each be greater than 8.");
    if (!(way_span > 0.0f))
        return set_err(BM_ERR_INVALID, "ScalarSdrWriter::new(): Waypoint span ('way_span') must be greater than zero.");
    if (!(lo <= hi)) return set_err(BM_ERR_INVALID, "ScalarSdrWriter::new(): empty value range");
    volatile float span = hi - lo;
    volatile float norm = span / way_span;
    const double ways = std::ceil((double)norm) + 1.0;
    const uint64_t len = (uint64_t)v_size * u_size;
    const uint64_t active = len / kSdrSparsity;
    if (ways > 65536.0 || active > 65535 || len > 0xFFFFFFFFull)
        return set_err(BM_ERR_UNSUPPORTED, "ScalarSdrWriter: too many waypoints or active axons");
    bm_sdr_writer_s* W = new (std::nothrow) bm_sdr_writer_s;
    if (!W) return set_err(BM_ERR_OOM, "host allocation failed");
    W->ctx = ctx;
    ctx_retain(ctx);
    W->lo = lo;
    W->hi = hi;
    W->way_span = way_span;
    W->len = (uint32_t)len;
    W->active = (uint32_t)active;
    W->way_count = (uint32_t)ways;
    // gen_axn_idxs (scalar_sdr_writer.rs:18-21): `active` uniform indices in
    // [0, len) per waypoint, repeats allowed, from a seeded stream.
    std::vector<uint32_t> idx((size_t)W->way_count * W->active);
    const uint64_t key = splitmix(seed ^ 0x7364727761797370ull);
    for (size_t k = 0; k < idx.size(); k++)
        idx[k] = (uint32_t)(((unsigned __int128)splitmix(key + k) * len) >> 64);
    DevGuard g(ctx->device);
    cudaError_t e = cudaSuccess;
    if (!idx.empty()) {
        e = cudaMalloc(&W->ways, idx.size() * sizeof(uint32_t));
        if (e == cudaSuccess) e = cudaMemcpy(W->ways, idx.data(), idx.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        if (W->ways) cudaFree(W->ways);
        ctx_release(W->ctx);
        delete W;
        return cuda_err(e, "sdr writer waypoints");
    }
    *out = W;
    return BM_OK;
}

int bm_sdr_writer_destroy(bm_sdr_writer w) {
    if (!w) return BM_OK;
    DevGuard g(w->ctx->device);
    if (w->ways) {
        cudaStreamSynchronize(w->ctx->stream());
        cudaFree(w->ways);
    }
    ctx_release(w->ctx);
    delete w;
    return BM_OK;
}

int bm_sdr_writer_info(bm_sdr_writer w, uint32_t* way_count, uint32_t* active, uint32_t* len) {
    if (!w) return set_err(BM_ERR_INVALID, "null writer");
    if (way_count) *way_count = w->way_count;
    if (active) *active = w->active;
    if (len) *len = w->len;
    return BM_OK;
}

int bm_sdr_writer_waypoints(bm_sdr_writer w, uint32_t* dst, uint64_t n) {
    if (!w || !dst) return set_err(BM_ERR_INVALID, "null argument");
    if (n != (uint64_t)w->way_count * w->active) return set_err(BM_ERR_INVALID, "waypoint table is %llu entries",
                                                                 (unsigned long long)w->way_count * w->active);
    DevGuard g(w->ctx->device);
    if (n) {
        const cudaError_t e = cudaMemcpy(dst, w->ways, n * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_err(e, "waypoints");
    }
    return BM_OK;
}

int bm_sdr_writer_encode(bm_sdr_writer w, const float* vals, uint32_t n, uint8_t* frames, uint64_t frame_stride) {
    if (!w || (n && (!vals || !frames))) return set_err(BM_ERR_INVALID, "null argument");
    if (n > kMaxEncodeValues / 2)
        return set_err(BM_ERR_INVALID, "sdr writer: at most %u values per call", kMaxEncodeValues / 2);
    if (frame_stride < w->len) return set_err(BM_ERR_INVALID, "sdr writer: frame stride below the frame's %u bytes", w->len);
    SdrArgs* A = new (std::nothrow) SdrArgs;
    if (!A) return set_err(BM_ERR_OOM, "host allocation failed");
    std::memset(A, 0, sizeof *A);
    A->n = n;
    for (uint32_t k = 0; k < n; k++) {
        // ScalarSdrWriter::encode (scalar_sdr_writer.rs:156-210) in f32.
        const float val = vals[k];
        if (!(val >= w->lo && val <= w->hi)) {
            delete A;
            return set_err(BM_ERR_INVALID, "ScalarSdrWriter::to_norm: Value (%g) out of range ((%g, %g)).", (double)val,
                           (double)w->lo, (double)w->hi);
        }
        volatile float d = val - w->lo;
        volatile float norm = d / w->way_span;
        volatile float way_0 = std::floor((float)norm);
        volatile float ratio = norm - way_0;
        volatile float cnt = (float)w->active * ratio;
        const uint32_t c1 = (uint32_t)cnt;
        const uint32_t i0 = (uint32_t)way_0;
        // The reference indexes the waypoint after way 0 even when it
        // contributes nothing, and panics past the last one.
        if (i0 + 1 >= w->way_count) {
            delete A;
            return set_err(BM_ERR_INVALID, "ScalarSdrWriter::encode: value %g needs waypoint %u of %u", (double)val, i0 + 1,
                           w->way_count);
        }
        A->way0[k] = i0;
        A->w0[k] = (uint16_t)(w->active - c1);
        A->w1[k] = (uint16_t)c1;
    }
    int rc = BM_OK;
    if (n) {
        DevGuard g(w->ctx->device);
        k_encode_sdr<<<n, 256, 0, w->ctx->stream()>>>(*A, w->ways, w->active, frames, frame_stride, w->len);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_err(e, "sdr writer");
    }
    delete A;
    return rc;
}

}  // extern "C"
