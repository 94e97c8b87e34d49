// bm_plain.cu -- the plain CUDA form of bismit's cycle: one kernel per
// reference stage, one area per launch, same stage order as the reference host.
// Each kernel restates the bismit OpenCL kernel it names; the fused stage
// kernels (bm_fused.cu) must produce identical bytes.
#include "bm_items.cuh"
#include "bm_kernels.h"

namespace bm {

namespace {

__device__ __forceinline__ uint64_t gtid() { return (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; }

// tft_set_syn_flags, cl/syns.cl:23-33, 16 synapses per thread.
__global__ void k_set_syn_flags(const uint8_t* __restrict__ states, uint8_t* __restrict__ flags, uint64_t n) {
    pdl_begin();
    uint64_t i = gtid() * 16;
    if (i + 16 <= n && ((((uintptr_t)states) | ((uintptr_t)flags)) & 15) == 0) {
        uint4 s = *(const uint4*)(states + i);
        uint4 f = *(const uint4*)(flags + i);
        uint32_t* sp = (uint32_t*)&s;
        uint32_t* fp = (uint32_t*)&f;
#pragma unroll
        for (int w = 0; w < 4; w++) {
            uint32_t x = sp[w];
            uint32_t nz = (((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x) & 0x80808080u;  // 0x80 per nonzero byte
            fp[w] = (fp[w] & 0xEFEFEFEFu) | (nz >> 3);
        }
        *(uint4*)(flags + i) = f;
    } else {
        for (uint64_t k = i; k < n && k < i + 16; k++)
            flags[k] = (uint8_t)((flags[k] & ~kSynPrevActiveFlag) | (states[k] ? kSynPrevActiveFlag : 0));
    }
}

// The per-item bodies are in bm_items.cuh; each kernel below is one area's
// stage, one thread per item.
__global__ void k_syn_cycle(const uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices,
                            DevLayer L, uint32_t t) {
    pdl_begin();
    uint64_t i = gtid();
    if (i >= (uint64_t)L.cells * L.tft[t].spt) return;
    syn_cycle_item(axns, slices, L, t, i);
}

__global__ void k_den_cycle(DevLayer L, uint32_t t, const AreaCtl* ctl) {
    pdl_begin();
    uint64_t d = gtid();
    if (d >= (uint64_t)L.cells * L.tft[t].dpt) return;
    den_cycle_item(L, t, rnd_at(L.tft[t].rnd_key_den, ctl->cycle), d);
}

__global__ void k_tft_cycle(DevLayer L, uint32_t t) {
    pdl_begin();
    uint32_t c = (uint32_t)gtid();
    if (c < L.cells) tft_cycle_item(L, t, c);
}

__global__ void k_ssc_cycle(DevLayer L) {
    pdl_begin();
    uint32_t c = (uint32_t)gtid();
    if (c < L.cells) ssc_cycle_item(L, c);
}

__global__ void k_inhib_simple(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices, DevLayer L,
                               int radius, uint64_t rnd_key, const AreaCtl* ctl) {
    pdl_begin();
    uint32_t c = (uint32_t)gtid();
    if (c < L.cells) inhib_simple_item(axns, slices, L, radius, rnd_at(rnd_key, ctl->cycle), c);
}

__global__ void k_inhib_passthrough(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices, DevLayer L) {
    pdl_begin();
    uint32_t c = (uint32_t)gtid();
    if (c < L.cells) inhib_passthrough_item(axns, slices, L, c);
}

__global__ void k_ssc_mtp_simple(const uint8_t* __restrict__ axns, DevLayer L, const AreaCtl* ctl) {
    pdl_begin();
    uint32_t c = (uint32_t)gtid();
    if (c < L.cells) ssc_mtp_item(axns, L, rnd_at(L.rnd_key_ssc_mtp, ctl->cycle), c);
}

__global__ void k_pyr_cycle(DevLayer L) {
    pdl_begin();
    uint32_t c = (uint32_t)gtid();
    if (c < L.cells) pyr_cycle_item(L, c);
}

__global__ void k_pyr_output(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices, DevLayer L) {
    pdl_begin();
    uint32_t c = (uint32_t)gtid();
    if (c < L.cells) pyr_output_item(axns, slices, L, c);
}

__global__ void k_inhib_intra_column(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices, DevLayer L) {
    pdl_begin();
    uint32_t col = (uint32_t)gtid();
    if (col < L.v_size * L.u_size) intra_column_item(axns, slices, L, col);
}

__global__ void k_tft_dst_mtp(const uint8_t* __restrict__ axns, DevLayer L, uint32_t t, const AreaCtl* ctl) {
    pdl_begin();
    uint32_t c = (uint32_t)gtid();
    if (c < L.cells) tft_dst_mtp_item(axns, L, t, rnd_at(L.tft[t].rnd_key_mtp, ctl->cycle), c);
}

__global__ void k_tuft_cells(const uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices, DevLayer L,
                             uint32_t t, const AreaCtl* ctl) {
    pdl_begin();
    uint32_t c = (uint32_t)gtid();
    if (c < L.cells) tuft_cell_item(axns, slices, L, t, rnd_at(L.tft[t].rnd_key_den, ctl->cycle), c);
}

// Warp-cooperative: no thread leaves before the warp's shared part. With
// host_cycle >= 0 the cycle number comes from the host (a launch on the
// area's front stream, which may run ahead of the area's counter).
__global__ void __launch_bounds__(128) k_inhib_mtp(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices,
                                                   DevLayer L, int radius, uint64_t key, int learn,
                                                   const AreaCtl* ctl, long long host_cycle) {
    pdl_begin();
    uint32_t c = (uint32_t)gtid();
    const unsigned long long cyc = host_cycle >= 0 ? (unsigned long long)host_cycle : ctl->cycle;
    inhib_mtp_warp(axns, slices, L, radius, rnd_at(key, cyc), rnd_at(L.rnd_key_ssc_mtp, cyc), learn != 0, c,
                   c < L.cells);
}

// With end_cycle, the last block to finish also ends the cycle (the cycle-end
// launch folded in): every block has read the cycle number by then. Twelve
// blocks of 128 per SM (40 registers): area_256's 262,144 cells then need 1.15
// waves of warps instead of the 1.54 that 54 registers allowed.
__global__ void __launch_bounds__(128, 12) k_pyr_tail(uint8_t* __restrict__ axns, const SliceRec* __restrict__ slices,
                                                  DevLayer L, int ctrl, int learn, AreaCtl* ctl, uint32_t tufts,
                                                  int end) {
    pdl_begin();
    const uint64_t i = gtid();
    pyr_tail_warp(axns, slices, L, ctrl, learn != 0, ctl, (uint32_t)i, i < tail_items(L.depth, L.v_size * L.u_size),
                  tufts);
    if (!end) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&ctl->blocks_done, 1u) == gridDim.x - 1) {
            ctl->blocks_done = 0;
            end_cycle(ctl);
        }
    }
}

inline unsigned nblk(uint64_t n, unsigned b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

// ------------------------------------------------------------ launchers ---
void launch_set_syn_flags(const DevLayer& L, cudaStream_t s) {
    uint64_t n = L.n_syns;
    if (!n) return;
    launch_pdl(k_set_syn_flags, nblk((n + 15) / 16, 256), 256, 0, s, L.buf[BM_BUF_SYN_STATES], L.buf[BM_BUF_SYN_FLAG_SETS], n);
}
void launch_set_syn_flags_tuft(const DevLayer& L, uint32_t t, cudaStream_t s) {
    const DevTuft& T = L.tft[t];
    uint64_t n = (uint64_t)L.cells * T.spt;
    if (!n) return;
    launch_pdl(k_set_syn_flags, nblk((n + 15) / 16, 256), 256, 0, s, L.buf[BM_BUF_SYN_STATES] + T.syn_idz,
                                                              L.buf[BM_BUF_SYN_FLAG_SETS] + T.syn_idz, n);
}
void launch_syn_cycle_plain(const uint8_t* axns, const SliceRec* slices, const DevLayer& L, uint32_t t,
                            cudaStream_t s) {
    uint64_t n = (uint64_t)L.cells * L.tft[t].spt;
    launch_pdl(k_syn_cycle, nblk(n, 256), 256, 0, s, axns, slices, L, t);
}
void launch_den_cycle_plain(const DevLayer& L, uint32_t t, const AreaCtl* ctl, cudaStream_t s) {
    uint64_t n = (uint64_t)L.cells * L.tft[t].dpt;
    launch_pdl(k_den_cycle, nblk(n, 256), 256, 0, s, L, t, ctl);
}
void launch_tft_cycle_plain(const DevLayer& L, uint32_t t, cudaStream_t s) {
    launch_pdl(k_tft_cycle, nblk(L.cells, 256), 256, 0, s, L, t);
}
void launch_ssc_cycle(const DevLayer& L, cudaStream_t s) {
    launch_pdl(k_ssc_cycle, nblk(L.cells, 256), 256, 0, s, L);
}
void launch_inhib_simple(uint8_t* axns, const SliceRec* slices, const DevLayer& L, int radius, uint64_t key,
                         const AreaCtl* ctl, cudaStream_t s) {
    launch_pdl(k_inhib_simple, nblk(L.cells, 128), 128, 0, s, axns, slices, L, radius, key, ctl);
}
void launch_inhib_passthrough(uint8_t* axns, const SliceRec* slices, const DevLayer& L, cudaStream_t s) {
    launch_pdl(k_inhib_passthrough, nblk(L.cells, 256), 256, 0, s, axns, slices, L);
}
void launch_ssc_mtp_plain(const uint8_t* axns, const DevLayer& L, const AreaCtl* ctl, cudaStream_t s) {
    launch_pdl(k_ssc_mtp_simple, nblk(L.cells, 128), 128, 0, s, axns, L, ctl);
}
void launch_pyr_cycle_plain(const DevLayer& L, cudaStream_t s) {
    launch_pdl(k_pyr_cycle, nblk(L.cells, 256), 256, 0, s, L);
}
void launch_pyr_output(uint8_t* axns, const SliceRec* slices, const DevLayer& L, cudaStream_t s) {
    launch_pdl(k_pyr_output, nblk(L.cells, 256), 256, 0, s, axns, slices, L);
}
// smooth_activity (cl/control.cl:227-295), one lattice of group centers: each
// center scans the hexagon of side r around it over every slice of the host
// layer (slice, then v offset, then u offset, as the reference loops), keeps
// the least active cell (ties: the later one) and the most active (ties: the
// later one), then raises the least active cell's energy by one and lowers
// the most active's by one, each within 0..255 and only when they differ.
// The groups of one lattice do not overlap, so the centers of a launch touch
// disjoint cells.
__global__ void k_smooth(DevLayer L, const int32_t* __restrict__ centers, uint32_t n, int32_t r) {
    pdl_begin();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t cv = centers[i] >> 16, cu = (int32_t)(int16_t)(centers[i] & 0xFFFF);
    const uint8_t* act = L.buf[BM_BUF_CEL_ACTIVITIES];
    uint8_t* en = L.buf[BM_BUF_CEL_ENERGIES];
    const int32_t vs = (int32_t)L.v_size, us = (int32_t)L.u_size;
    uint32_t least_idx = 0, most_idx = 0;
    uint32_t least_act = 255, most_act = 0;
    for (uint32_t slc = 0; slc < L.depth; slc++)
        for (int32_t vo = -r; vo <= r; vo++) {
            const int32_t uz = max(-r, -vo - r), um = min(r, -vo + r);
            const int32_t v = cv + vo;
            for (int32_t uo = uz; uo <= um; uo++) {
                const int32_t u = cu + uo;
                if (v < 0 || v >= vs || u < 0 || u >= us) continue;
                const uint32_t idx = slc * (uint32_t)(vs * us) + (uint32_t)(v * us + u);
                const uint32_t a = act[idx];
                if (a <= least_act) { least_idx = idx; least_act = a; }
                if (a >= most_act) { most_idx = idx; most_act = a; }
            }
        }
    // Equal indices change nothing; skipping the write matters, because a
    // hexagon wholly outside the layer leaves both at cell 0, and writing
    // cell 0's energy back would race the one hexagon of the lattice that
    // holds cell 0.
    if (least_idx == most_idx) return;
    const uint32_t le = en[least_idx];
    en[least_idx] = (uint8_t)(le + (uint32_t)((le < 255) & (most_act < 255)));
    const uint32_t me = en[most_idx];
    en[most_idx] = (uint8_t)(me - (uint32_t)((me > 0) & (most_act > 0)));
}

void launch_smooth(const DevLayer& L, const int32_t* centers, uint32_t n, int32_t radius, cudaStream_t s) {
    if (n) launch_pdl(k_smooth, nblk(n, 128), 128, 0, s, L, centers, n, radius);
}

// retina (cl/filters.cl:34-100), one input filter over a (depth, v, u) grid
// of input bytes. Cell i (its index in the grid) is an off-center cell when
// bit 0 of i is set and a large one when bits 1 and 0 differ; it averages the
// hexagon of radius 5 (large) or 3 (small) around it in its own slice,
// counting cells outside the grid as zero but still dividing by the full
// hexagon (get_neighbors_avg, :8-31). The output is how far the average
// exceeds the cell by more than RETNAL_THRESHOLD (48, cl/bismit.cl:19) for an
// off-center cell, or the cell the average, else 0. It goes to slice
// base_slc + slice of the output at that slice's first axon (the slice
// table's x), the cell's (v, u) place within the slice.
__global__ void k_retina(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, const SliceRec* __restrict__ slices,
                         uint32_t base_slc, uint32_t depth, uint32_t vs, uint32_t us) {
    pdl_begin();
    const uint32_t cols = vs * us;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= depth * cols) return;
    const uint32_t slc = i / cols, col = i - slc * cols;
    const int32_t v = (int32_t)(col / us), u = (int32_t)(col - (uint32_t)v * us);
    const uint8_t* plane = in + (uint64_t)slc * cols;
    const uint32_t off_cen = i & 1, large = ((i & 3) >> 1) ^ off_cen;
    const int32_t r = large ? 5 : 3;
    int32_t sum = 0;
    for (int32_t vo = -r; vo <= r; vo++) {
        const int32_t vv = v + vo;
        if (vv < 0 || vv >= (int32_t)vs) continue;
        const int32_t uz = max(-r, -vo - r), um = min(r, -vo + r);
        const uint8_t* row = plane + (uint32_t)vv * us;
        for (int32_t uo = uz; uo <= um; uo++) {
            const int32_t uu = u + uo;
            if (uu >= 0 && uu < (int32_t)us) sum += row[uu];
        }
    }
    const int32_t avg = sum / (3 * r * r + 3 * r + 1);
    const int32_t center = in[i];
    int32_t st;
    if (off_cen) {
        const int32_t cst = center + kRetinalThreshold;
        st = avg > cst ? avg - cst : 0;
    } else {
        const int32_t nat = avg + kRetinalThreshold;
        st = center > nat ? center - nat : 0;
    }
    out[slices[(base_slc + slc) & 0xFF].x + col] = (uint8_t)st;
}

void launch_retina(const uint8_t* in, uint8_t* out, const SliceRec* slices, uint32_t base_slc, uint32_t depth,
                   uint32_t v_size, uint32_t u_size, cudaStream_t s) {
    const uint32_t n = depth * v_size * u_size;
    if (n) launch_pdl(k_retina, nblk(n, 256), 256, 0, s, in, out, slices, base_slc, depth, v_size, u_size);
}

void launch_inhib_intra_column_plain(uint8_t* axns, const SliceRec* slices, const DevLayer& L, cudaStream_t s) {
    launch_pdl(k_inhib_intra_column, nblk((uint64_t)L.v_size * L.u_size, 256), 256, 0, s, axns, slices, L);
}
void launch_tuft_cells(const uint8_t* axns, const SliceRec* slices, const DevLayer& L, uint32_t t,
                       const AreaCtl* ctl, cudaStream_t s) {
    launch_pdl(k_tuft_cells, nblk(L.cells, 128), 128, 0, s, axns, slices, L, t, ctl);
}
void launch_inhib_mtp(uint8_t* axns, const SliceRec* slices, const DevLayer& L, int radius, uint64_t key,
                      bool learn, const AreaCtl* ctl, cudaStream_t s, int64_t host_cycle) {
    launch_pdl(k_inhib_mtp, nblk(L.cells, 128), 128, 0, s, axns, slices, L, radius, key, learn ? 1 : 0, ctl,
               (long long)host_cycle);
}
void launch_pyr_tail(uint8_t* axns, const SliceRec* slices, const DevLayer& L, int ctrl, bool learn, AreaCtl* ctl,
                     cudaStream_t s, uint32_t tufts, bool end) {
    launch_pdl(k_pyr_tail, nblk(tail_items(L.depth, L.v_size * L.u_size), 128), 128, 0, s, axns, slices, L, ctrl,
               learn ? 1 : 0, ctl, tufts, end ? 1 : 0);
}
void launch_tft_dst_mtp_plain(const uint8_t* axns, const DevLayer& L, uint32_t t, const AreaCtl* ctl,
                              cudaStream_t s) {
    launch_pdl(k_tft_dst_mtp, nblk(L.cells, 128), 128, 0, s, axns, L, t, ctl);
}

}  // namespace bm
