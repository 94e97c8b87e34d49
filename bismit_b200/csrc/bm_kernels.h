// bm_kernels.h -- host-callable launchers of the cycle kernels.
#pragma once
#include "bm_dev.cuh"

namespace bm {

// Growth parameters of one tuft (see bm_grow.cu).
struct GrowTuft {
    uint32_t tft;
    uint64_t key;
    uint32_t n_pool;                          // pool with prevalence repeats
    uint8_t pool[BM_MAX_SRC_SLICES];          // slice id per pool entry
    uint8_t pool_src[BM_MAX_SRC_SLICES];      // index of the pool entry's distinct source
    uint8_t nonspatial[BM_MAX_SRC_SLICES];
    int32_t rv[BM_MAX_SRC_SLICES], ru[BM_MAX_SRC_SLICES];   // scaled reaches / nonspatial half sizes
    uint32_t n_offs[BM_MAX_SRC_SLICES];
    uint32_t offs_base[BM_MAX_SRC_SLICES];
    const int8_t* offs_v;
    const int8_t* offs_u;
    uint32_t unique, zero_strength;
};

// Stores the calling thread's error message (bm_last_error) and returns `code`.
int set_err(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
// Device view of data layer i of a state slab laid out by plan P.
void fill_dev_layer(DevLayer& D, const bm_area_plan& P, uint32_t i, uint8_t* slab);
// Device slice records of plan P, BM_MAX_SLICES entries (zero past n_slices).
void fill_slice_table(const bm_area_plan& P, SliceRec* out);

void launch_grow(const DevLayer& L, const GrowTuft& G, cudaStream_t s);

// Regrowth (bm_grow.cu) acts on the cycles c with c % kRegrowPeriod ==
// kRegrowPeriod - 1: bismit's counter (src/cortex/cortical_area.rs:792-806)
// counts up from 0 and fires, resetting, once it has reached
// SYNAPSE_REGROWTH_INTERVAL (200, src/cmn/mod.rs:234).
constexpr uint32_t kRegrowPeriod = 201;
constexpr int kStrengthFloor = -25;   // SYNAPSE_STRENGTH_FLOOR, src/cmn/mod.rs:233
constexpr uint32_t kRegrowBlock = 128;

// Gather geometry of a tiled tuft. Its cells are cut into tiles of tile_h
// rows x tile_w columns of one layer slice; a tile's footprint holds, for each
// of the nrec source slices from slc0 on, the rows and columns its cells'
// scaled positions reach with offsets up to rv, ru (rows of fw bytes, fsz
// bytes per slice). With xalign the footprint is loaded by the tensor memory
// accelerator, whose boxes start on a 16-byte column boundary: each row then
// begins at the tile's first column rounded down to a multiple of 16, and
// every column sits (first column & 15) bytes further in.
struct GatherGeo {
    uint32_t S_l2;           // log2 synapses per cell-tuft
    uint32_t cols, u_size;   // layer columns, row width
    uint32_t tile_w, tile_h;
    uint32_t vs, us;         // scale of the source slices (shared by all of them)
    int32_t rv, ru;
    uint32_t fw, fsz;
    uint32_t slc0, nrec;
    uint32_t xalign;
};

// The byte that the synapse at tuft offset i with source (slc, v_ofs, u_ofs)
// gathers, as an offset into its tile's footprint; false (and 0) when the
// footprint does not hold it. The tile's footprint starts (rv, ru) before its
// first cell's scaled position, so a cell at (v, u) in the tile with origin
// (v0, u0) reads row (v*vs >> 4) - (v0*vs >> 4) + rv + v_ofs.
__host__ __device__ __forceinline__ uint32_t gather_offset(const GatherGeo& g, uint64_t i, uint32_t slc, int vo,
                                                           int uo, bool& ok) {
    const uint32_t c = (uint32_t)(i >> g.S_l2);
    const uint32_t rem = c % g.cols;
    const uint32_t v = rem / g.u_size, u = rem - (rem / g.u_size) * g.u_size;
    const uint32_t v0 = v - v % g.tile_h, u0 = u - u % g.tile_w;
    const int32_t ulo = (int32_t)((u0 * g.us) >> 4) - g.ru;   // the footprint's first column
    const int32_t row = (int32_t)((v * g.vs) >> 4) - (int32_t)((v0 * g.vs) >> 4) + g.rv + vo;
    const int32_t col = (int32_t)((u * g.us) >> 4) - ulo + uo + (g.xalign ? (ulo & 15) : 0);
    const uint32_t k = slc - g.slc0;
    ok = k < g.nrec && vo >= -g.rv && vo <= g.rv && uo >= -g.ru && uo <= g.ru;
    return ok ? k * g.fsz + (uint32_t)row * g.fw + (uint32_t)col : 0u;
}

// Gather geometry of a tiled tuft as regrowth needs it (regrowth recompiles
// the offsets of the synapses it moves); kept current in device memory across
// retiling.
struct TuftGeo {
    uint16_t* gidx;          // null: the tuft is not tiled
    GatherGeo g;
    uint32_t tiled;
};

// Regrowth of one tuft of one area: one thread per dendrite.
struct RegrowJob {
    DevLayer L;
    GrowTuft G;              // the tuft's pools (offset arrays kept by the area)
    const AreaCtl* ctl;
    const TuftGeo* geo;
    uint64_t rkey;           // stream key; round r = c / kRegrowPeriod draws from splitmix64(rkey + r)
    uint32_t saturated;      // the pool is saturated: the first draw is kept
    uint32_t n;              // dendrites
    uint32_t block0;         // first block of this job in its launch
};
uint64_t regrow_key(uint64_t grow_key);
void launch_regrow(const RegrowJob* jobs, uint32_t n_jobs, uint32_t n_blocks, cudaStream_t s);
void launch_cycle_end(AreaCtl* ctl, cudaStream_t s);
// Device-to-device copies of a frame's pieces as one programmatic-dependent
// launch: on the cycling stream it chains with the cycle's kernels, where a
// memcpy would end the chain (the next kernel could only start once the copy
// had completed).
constexpr uint32_t kMaxCopyPieces = 8;
struct CopyPieces {
    uint8_t* dst[kMaxCopyPieces];
    const uint8_t* src[kMaxCopyPieces];
    uint32_t len[kMaxCopyPieces];
    uint32_t n;
};
void launch_copy_pieces(const CopyPieces& P, cudaStream_t s);

// Plain form: one kernel per reference stage (bm_plain.cu).
void launch_set_syn_flags(const DevLayer& L, cudaStream_t s);
void launch_set_syn_flags_tuft(const DevLayer& L, uint32_t t, cudaStream_t s);
void launch_syn_cycle_plain(const uint8_t* axns, const SliceRec* slices, const DevLayer& L, uint32_t t,
                            cudaStream_t s);
void launch_den_cycle_plain(const DevLayer& L, uint32_t t, const AreaCtl* ctl, cudaStream_t s);
void launch_tft_cycle_plain(const DevLayer& L, uint32_t t, cudaStream_t s);
void launch_ssc_cycle(const DevLayer& L, cudaStream_t s);
void launch_inhib_simple(uint8_t* axns, const SliceRec* slices, const DevLayer& L, int radius, uint64_t key,
                         const AreaCtl* ctl, cudaStream_t s);
void launch_inhib_passthrough(uint8_t* axns, const SliceRec* slices, const DevLayer& L, cudaStream_t s);
void launch_ssc_mtp_plain(const uint8_t* axns, const DevLayer& L, const AreaCtl* ctl, cudaStream_t s);
void launch_pyr_cycle_plain(const DevLayer& L, cudaStream_t s);
void launch_pyr_output(uint8_t* axns, const SliceRec* slices, const DevLayer& L, cudaStream_t s);
void launch_inhib_intra_column_plain(uint8_t* axns, const SliceRec* slices, const DevLayer& L, cudaStream_t s);
// One lattice of the activity smoother's group centers (bm_plain.cu).
void launch_smooth(const DevLayer& L, const int32_t* centers, uint32_t n, int32_t radius, cudaStream_t s);
// One retina filter (cl/filters.cl:34-100) from a (depth, v_size, u_size)
// input grid to slices base_slc.. of `out`, each at its slice-table offset.
void launch_retina(const uint8_t* in, uint8_t* out, const SliceRec* slices, uint32_t base_slc, uint32_t depth,
                   uint32_t v_size, uint32_t u_size, cudaStream_t s);
// Fused cell steps (bm_items.cuh): an unfused tuft's four stages per cell;
// inhibition with spiny stellate learning; pyramidal soma, control and distal
// learning per column (ctrl: 0 none, 1 intra-column, 2 output).
void launch_tuft_cells(const uint8_t* axns, const SliceRec* slices, const DevLayer& L, uint32_t t,
                       const AreaCtl* ctl, cudaStream_t s);
void launch_inhib_mtp(uint8_t* axns, const SliceRec* slices, const DevLayer& L, int radius, uint64_t key,
                      bool learn, const AreaCtl* ctl, cudaStream_t s, int64_t host_cycle = -1);
// `tufts` (bit t): tufts the fused tuft kernel does not take, run per cell
// first; `end`: the last block to finish also ends the cycle.
void launch_pyr_tail(uint8_t* axns, const SliceRec* slices, const DevLayer& L, int ctrl, bool learn, AreaCtl* ctl,
                     cudaStream_t s, uint32_t tufts = 0, bool end = false);
void launch_tft_dst_mtp_plain(const uint8_t* axns, const DevLayer& L, uint32_t t, const AreaCtl* ctl,
                              cudaStream_t s);

}  // namespace bm
