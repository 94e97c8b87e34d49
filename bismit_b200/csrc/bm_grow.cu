// bm_grow.cu -- on-device synapse growth and small control kernels.
//
// Growth restates Synapses::grow(init = true) (src/cortex/synapses.rs:454-501)
// with SynSrcSlices::gen_src (src/map/syn_src.rs:448-490) and the per-dendrite
// uniqueness rule of SynSrcIdxCache::insert (src/map/syn_src.rs:186-203). The
// entropy-seeded SmallRng is replaced by a seeded per-dendrite counter stream,
// so one thread grows one dendrite and the result does not depend on launch
// order. The same rule is restated in the oracle (bmo_grow).
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

__global__ void k_grow(DevLayer L, GrowTuft G) {
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
    for (uint32_t j = 0; j < T.spd; j++) {
        uint8_t ns = 0;
        int nv = 0, nu = 0, nstr = 0;
        for (int att = 0; att < kGrowMaxAttempts; att++) {
            uint64_t w = grow_word(G.key, d, wk++);
            uint64_t w2 = grow_word(G.key, d, wk++);
            uint32_t pi = uniform_idx((uint32_t)w, G.n_pool);
            ns = G.pool[pi];
            uint32_t k = G.pool_src[pi];
            if (G.nonspatial[k]) {
                nv = (int)uniform_idx((uint32_t)(w >> 32), (uint32_t)(2 * G.rv[k] + 1)) - G.rv[k];
                nu = (int)uniform_idx((uint32_t)w2, (uint32_t)(2 * G.ru[k] + 1)) - G.ru[k];
                nstr = 0;
            } else {
                uint32_t oi = uniform_idx((uint32_t)(w >> 32), G.n_offs[k]);
                nv = G.offs_v[G.offs_base[k] + oi];
                nu = G.offs_u[G.offs_base[k] + oi];
                int inten = ((G.rv[k] - abs(nv)) + (G.ru[k] - abs(nu))) >> 3;
                int r = (int)uniform_idx((uint32_t)w2, 7u) - 3;
                nstr = (int)(int8_t)(uint8_t)(inten * r);
            }
            if (!G.unique) break;
            int64_t nk = (int64_t)ns * cols + (int64_t)nv * L.u_size + nu;
            if (nk == 0) break;  // key 0 is never retained (old-source removal at init)
            bool dup = false;
            for (uint32_t jj = 0; jj < j; jj++) {
                int64_t ok = (int64_t)slc[s0 + jj] * cols + (int64_t)vo[s0 + jj] * L.u_size + uo[s0 + jj];
                if (ok == nk) { dup = true; break; }
            }
            if (!dup) break;
        }
        slc[s0 + j] = ns;
        vo[s0 + j] = (int8_t)nv;
        uo[s0 + j] = (int8_t)nu;
        str[s0 + j] = G.zero_strength ? (int8_t)0 : (int8_t)nstr;
    }
}

__global__ void k_cycle_end(AreaCtl* ctl) { ctl->cycle += 1; }

}  // namespace

void launch_grow(const DevLayer& L, const GrowTuft& G, cudaStream_t s) {
    uint64_t n = (uint64_t)L.cells * L.tft[G.tft].dpt;
    k_grow<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(L, G);
}

void launch_cycle_end(AreaCtl* ctl, cudaStream_t s) { k_cycle_end<<<1, 1, 0, s>>>(ctl); }

}  // namespace bm
