// bm_grow.cu -- on-device synapse growth and small control kernels.
//
// Growth restates Synapses::grow(init = true) (src/cortex/synapses.rs:454-501)
// with SynSrcSlices::gen_src (src/map/syn_src.rs:448-490) and the per-dendrite
// uniqueness rule of SynSrcIdxCache::insert (src/map/syn_src.rs:186-203). The
// entropy-seeded SmallRng is replaced by a seeded per-dendrite counter stream,
// so one thread grows one dendrite and the result does not depend on launch
// order. The same rule is restated in the oracle (bmo_grow). Regrowth
// (k_regrow) draws from the same pools with a per-round stream.
#include <algorithm>

#include "bm_kernels.h"

namespace bm {

namespace {

__device__ __forceinline__ uint64_t grow_word(uint64_t key, uint64_t den, uint64_t k) {
    return splitmix64(splitmix64(key + den) + k);
}
__device__ __forceinline__ uint32_t uniform_idx(uint32_t r, uint32_t n) {
    return (uint32_t)(((uint64_t)r * n) >> 32);
}

constexpr int kGrowMaxAttempts = 1024;

// One candidate source from two words of a dendrite's stream
// (SynSrcSlices::gen_src, src/map/syn_src.rs:448-490): a uniform pick of the
// tuft's source slices, then of that slice's offset pool (or of its whole
// grid for a nonspatial slice), and a strength of intensity x U[-3, 3] where
// intensity is the scaled reach left over by the offset, >> 3.
__device__ __forceinline__ void draw_src(const GrowTuft& G, uint64_t w, uint64_t w2, uint8_t& ns, int& nv, int& nu,
                                         int& nstr) {
    const uint32_t pi = uniform_idx((uint32_t)w, G.n_pool);
    ns = G.pool[pi];
    const uint32_t k = G.pool_src[pi];
    if (G.nonspatial[k]) {
        nv = (int)uniform_idx((uint32_t)(w >> 32), (uint32_t)(2 * G.rv[k] + 1)) - G.rv[k];
        nu = (int)uniform_idx((uint32_t)w2, (uint32_t)(2 * G.ru[k] + 1)) - G.ru[k];
        nstr = 0;
    } else {
        const uint32_t oi = uniform_idx((uint32_t)(w >> 32), G.n_offs[k]);
        nv = G.offs_v[G.offs_base[k] + oi];
        nu = G.offs_u[G.offs_base[k] + oi];
        const int inten = ((G.rv[k] - abs(nv)) + (G.ru[k] - abs(nu))) >> 3;
        const int r = (int)uniform_idx((uint32_t)w2, 7u) - 3;
        nstr = (int)(int8_t)(uint8_t)(inten * r);
    }
}

// Dendrites of up to this many synapses keep their drawn sources' keys in
// shared memory for the uniqueness test (one row per thread, padded against
// bank conflicts; 32-bit while the keys fit, below 2^31); longer ones, or
// grids too large for those keys, read the sources back from the slab.
constexpr uint32_t kGrowKeys = 64;
constexpr uint32_t kGrowBlock = 128;

__global__ void __launch_bounds__(kGrowBlock) k_grow(DevLayer L, GrowTuft G) {
    __shared__ int32_t keys[kGrowBlock][kGrowKeys + 1];
    uint64_t d = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const DevTuft& T = L.tft[G.tft];
    uint64_t n_dens = (uint64_t)L.cells * T.dpt;
    if (d >= n_dens) return;
    uint8_t* slc = L.buf[BM_BUF_SYN_SRC_SLC_IDS];
    int8_t* vo = (int8_t*)L.buf[BM_BUF_SYN_SRC_COL_V_OFFS];
    int8_t* uo = (int8_t*)L.buf[BM_BUF_SYN_SRC_COL_U_OFFS];
    int8_t* str = (int8_t*)L.buf[BM_BUF_SYN_STRENGTHS];
    int64_t cols = (int64_t)L.v_size * L.u_size;
    uint64_t s0 = T.syn_idz + d * T.spd;
    uint64_t wk = 0;
    const bool cached = T.spd <= kGrowKeys && cols < (1ll << 22);   // |key| < 382 * 2^22 < 2^31
    int32_t* my = keys[threadIdx.x];
    for (uint32_t j = 0; j < T.spd; j++) {
        uint8_t ns = 0;
        int nv = 0, nu = 0, nstr = 0;
        int64_t nk = 0;
        for (int att = 0; att < kGrowMaxAttempts; att++) {
            const uint64_t w = grow_word(G.key, d, wk++);
            const uint64_t w2 = grow_word(G.key, d, wk++);
            draw_src(G, w, w2, ns, nv, nu, nstr);
            nk = (int64_t)ns * cols + (int64_t)nv * L.u_size + nu;
            if (!G.unique) break;
            if (nk == 0) break;  // key 0 is never retained (old-source removal at init)
            bool dup = false;
            for (uint32_t jj = 0; jj < j; jj++) {
                const int64_t ok = cached ? (int64_t)my[jj]
                                          : (int64_t)slc[s0 + jj] * cols + (int64_t)vo[s0 + jj] * L.u_size + uo[s0 + jj];
                if (ok == nk) { dup = true; break; }
            }
            if (!dup) break;
        }
        if (cached) my[j] = (int32_t)nk;
        slc[s0 + j] = ns;
        vo[s0 + j] = (int8_t)nv;
        uo[s0 + j] = (int8_t)nu;
        str[s0 + j] = G.zero_strength ? (int8_t)0 : (int8_t)nstr;
    }
}

__global__ void k_cycle_end(AreaCtl* ctl) { pdl_begin(); end_cycle(ctl); }

// Piece blockIdx.y of P, 16 bytes a thread where both ends allow it.
__global__ void __launch_bounds__(256) k_copy_pieces(const __grid_constant__ CopyPieces P) {
    pdl_begin();
    const uint32_t k = blockIdx.y;
    uint8_t* dst = P.dst[k];
    const uint8_t* src = P.src[k];
    const uint32_t n = P.len[k];
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
    if ((((uintptr_t)dst | (uintptr_t)src) & 15) == 0) {
        const uint32_t n16 = n / 16;
        for (uint32_t i = t0; i < n16; i += stride) ((uint4*)dst)[i] = ((const uint4*)src)[i];
        for (uint32_t i = n16 * 16 + t0; i < n; i += stride) dst[i] = src[i];
    } else {
        for (uint32_t i = t0; i < n; i += stride) dst[i] = src[i];
    }
}

// Synapses::regrow (src/cortex/synapses.rs:411-501) with SynSrcIdxCache
// (src/map/syn_src.rs:159-211), one dendrite per thread, on the cycles c with
// c % kRegrowPeriod == kRegrowPeriod - 1 (other cycles return at once). Each
// synapse at or below the strength floor draws sources, in synapse order,
// until the dendrite's source set lacks the new key (slice * columns + v_ofs
// * u_size + u_ofs), or at once for a saturated pool. The set is every
// non-zero key of the dendrite's sources plus key 0 when den_src_key0 says so:
// bismit's cache inserts the new key and, if that was new, drops the old one,
// so an accepted key 0 enters unless the old key was 0, which always leaves.
// Draws stop after kGrowMaxAttempts, keeping the last. A tiled tuft's
// compiled gather offset follows each moved synapse. The same rule is
// restated in the oracle.
__global__ void __launch_bounds__(kRegrowBlock) k_regrow(const RegrowJob* __restrict__ jobs, uint32_t n_jobs) {
    pdl_begin();
    __shared__ uint32_t s_j;
    if (threadIdx.x == 0) {
        uint32_t lo = 0, hi = n_jobs;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (jobs[mid].block0 <= blockIdx.x) lo = mid;
            else hi = mid;
        }
        s_j = lo;
    }
    __syncthreads();
    const RegrowJob& J = jobs[s_j];
    const uint64_t cyc = J.ctl->cycle;
    if (cyc % kRegrowPeriod != kRegrowPeriod - 1) return;
    const uint32_t d = (blockIdx.x - J.block0) * kRegrowBlock + threadIdx.x;
    if (d >= J.n) return;
    const DevLayer& L = J.L;
    const DevTuft& T = L.tft[J.G.tft];
    uint8_t* slc = L.buf[BM_BUF_SYN_SRC_SLC_IDS];
    int8_t* vo = (int8_t*)L.buf[BM_BUF_SYN_SRC_COL_V_OFFS];
    int8_t* uo = (int8_t*)L.buf[BM_BUF_SYN_SRC_COL_U_OFFS];
    int8_t* str = (int8_t*)L.buf[BM_BUF_SYN_STRENGTHS];
    uint8_t* z = L.buf[BM_BUF_DEN_SRC_KEY0] + T.den_idz + d;
    const TuftGeo geo = *J.geo;
    const uint64_t rk = splitmix64(J.rkey + cyc / kRegrowPeriod);
    const int64_t cols = (int64_t)L.v_size * L.u_size;
    const uint64_t s0 = T.syn_idz + (uint64_t)d * T.spd;
    uint64_t wk = 0;
    for (uint32_t j = 0; j < T.spd; j++) {
        if (str[s0 + j] > kStrengthFloor) continue;
        const int64_t ko = (int64_t)slc[s0 + j] * cols + (int64_t)vo[s0 + j] * L.u_size + uo[s0 + j];
        uint8_t ns = 0;
        int nv = 0, nu = 0, nstr = 0;
        int64_t nk = 0;
        for (int att = 0; att < kGrowMaxAttempts; att++) {
            const uint64_t w = grow_word(rk, d, wk++);
            const uint64_t w2 = grow_word(rk, d, wk++);
            draw_src(J.G, w, w2, ns, nv, nu, nstr);
            nk = (int64_t)ns * cols + (int64_t)nv * L.u_size + nu;
            if (J.saturated) break;
            bool held;
            if (nk == 0) {
                held = *z != 0;
            } else {
                held = false;
                for (uint32_t jj = 0; jj < T.spd; jj++) {
                    const int64_t ok = (int64_t)slc[s0 + jj] * cols + (int64_t)vo[s0 + jj] * L.u_size + uo[s0 + jj];
                    if (ok == nk) { held = true; break; }
                }
            }
            if (!held) break;
        }
        if (!J.saturated) {
            if (ko == 0) *z = 0;
            else if (nk == 0) *z = 1;
        }
        slc[s0 + j] = ns;
        vo[s0 + j] = (int8_t)nv;
        uo[s0 + j] = (int8_t)nu;
        str[s0 + j] = (int8_t)nstr;
        // A tiled tuft's pools lie inside its footprint (every draw is held).
        if (geo.tiled) {
            bool ok;
            const uint64_t i = s0 + j - T.syn_idz;
            geo.gidx[i] = (uint16_t)gather_offset(geo.g, i, ns, nv, nu, ok);
        }
    }
}

}  // namespace

void launch_grow(const DevLayer& L, const GrowTuft& G, cudaStream_t s) {
    uint64_t n = (uint64_t)L.cells * L.tft[G.tft].dpt;
    k_grow<<<(unsigned)((n + kGrowBlock - 1) / kGrowBlock), kGrowBlock, 0, s>>>(L, G);
}

void launch_cycle_end(AreaCtl* ctl, cudaStream_t s) { launch_pdl(k_cycle_end, 1, 1, 0, s, ctl); }

void launch_copy_pieces(const CopyPieces& P, cudaStream_t s) {
    uint32_t most = 0;
    for (uint32_t k = 0; k < P.n; k++) most = std::max(most, P.len[k]);
    if (!most) return;
    const uint32_t blocks = std::min<uint32_t>(148, (most + 4095) / 4096);
    launch_pdl(k_copy_pieces, dim3(blocks, P.n), 256, 0, s, P);
}

uint64_t regrow_key(uint64_t gkey) { return splitmix64(gkey ^ 0x7265677277ull); }

void launch_regrow(const RegrowJob* jobs, uint32_t n_jobs, uint32_t n_blocks, cudaStream_t s) {
    if (n_blocks) launch_pdl(k_regrow, n_blocks, kRegrowBlock, 0, s, jobs, n_jobs);
}

}  // namespace bm
