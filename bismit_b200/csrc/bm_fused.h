// bm_fused.h -- the fused stage kernels: per-area preparation and launchers.
#pragma once
#include <string>
#include <vector>

#include "bm_dev.cuh"
#include "bm_kernels.h"
#include "bm_layout.h"

namespace bm {

// Launch parameters of the fused kernel for one tuft.
struct FusedTuft {
    bool ok = false;         // the fused kernel applies to this tuft
    uint32_t slc0 = 0;       // fast gathers serve slices slc0 .. slc0 + nrec - 1
    uint32_t nrec = 0;
    bool tiled = false;      // gathers from a shared-memory footprint
    uint32_t tile_w = 0, tile_h = 0;
    int32_t rv = 0, ru = 0;  // footprint margin: the pool's largest |v|, |u| offsets
    uint32_t fw = 0, frows = 0, fsz = 0;   // footprint width, rows, bytes per slice
    uint16_t* gidx = nullptr;   // compiled gather offsets, one per synapse of the tuft
    uint32_t smem = 0;       // dynamic shared memory per CTA
    uint32_t grid = 1;       // persistent grid size
    uint32_t nst = 2;        // TMA pipeline stages
    uint32_t stage_bytes = 0;
    uint32_t ring_off = 0;   // ring offset in dynamic shared memory (the footprint is at 0)
    uint32_t stage_stride = 0;   // bytes per ring buffer
    uint32_t win_bytes = 0;      // bytes per dendrite / cell-tuft window
    bool win = false;            // windows ride in the stages (16-byte aligned ranges)
    uint32_t src_vs = 0, src_us = 0, src_vsz = 0, src_usz = 0;
    uint32_t src_idz[8] = {};
    uint32_t tile_target = 0;    // synapses per tile asked for (0: chosen from the tuft's size)
    bool tile_tuned = false;     // tile_target came from the autotuner
    bool fp_staged = false;      // the consumers stage the footprint even where a tensor box could load it
                                 // (the autotuner's choice)
    // Footprint loaded by the tensor memory accelerator (a 3-D box of the
    // source slices) instead of staged by the consumer warps; rows of fw
    // bytes then start on a 16-byte column boundary (GatherGeo::xalign).
    bool fp_tma = false;
    alignas(64) unsigned char tmap[128] = {};   // its tensor map (bind_fused_tuft), a CUtensorMap
    const uint8_t* bound_axns = nullptr;        // the axon space the tensor map points into
};

struct FusedArea {
    int sms = 148;
    FusedTuft t[BM_MAX_LAYERS][BM_MAX_TUFTS];
    // Where the gather offsets come from: this pool in stream order on
    // pool_stream when set, else cudaMalloc.
    cudaMemPool_t pool = nullptr;
    cudaStream_t pool_stream = nullptr;
};

// Decides, per tuft, whether the fused kernel applies (syns_per_den a power of
// two in 16..512, dens_per_tft a power of two, 16-byte aligned ranges) and
// its gather form. Tufts that do not qualify run the plain per-stage kernels.
int prepare_fused(FusedArea& F, const bm_area_plan& P, std::string* err);
// The same decisions without allocating (gidx pointers left null), for every
// tuft of the area or for one.
int plan_fused(FusedArea& F, const bm_area_plan& P);
int plan_fused_tuft(FusedArea& F, const bm_area_plan& P, uint32_t layer, uint32_t t);
// Replans a tiled tuft for about `target_syns` synapses per tile, keeping its
// gather-offset buffer; `staged`: the consumers stage the footprint (no
// tensor box). False, and nothing changed, when the tuft would not stay
// tiled. *changed tells whether the tiles or the footprint form changed, in
// which case the caller recompiles the offsets before the next launch.
bool retile_fused_tuft(FusedArea& F, const bm_area_plan& P, uint32_t layer, uint32_t t, uint32_t target_syns,
                       bool* changed, bool staged = false);
// Frees the gather offsets (pooled ones in stream order on s).
void free_fused(FusedArea& F, cudaStream_t s = nullptr);
// Encodes the footprint tensor maps of the tufts that load their footprint
// with the tensor memory accelerator, for the axon space at `axns` (device
// memory, 16-byte aligned). BM_ERR_CUDA when the driver refuses one.
int bind_fused(FusedArea& F, const bm_area_plan& P, const uint8_t* axns);
int bind_fused_tuft(FusedArea& F, const bm_area_plan& P, uint32_t layer, uint32_t t, const uint8_t* axns);
// The specialised consumer shape tiled tuft FT's launches use while its flags
// are clean and its sources lie in the footprint (0: the general consumer).
uint32_t consumer_shape(const FusedTuft& FT, uint32_t spt, uint32_t spd, bool pyramidal);
// Gather geometry of tiled tuft t of data layer `layer` as planned in F.
GatherGeo gather_geo(const FusedArea& F, const bm_area_plan& P, uint32_t layer, uint32_t t);
// Synapse flags + synapse cycle + dendrite cycle (+ tuft cycle for pyramidal
// layers) of one tuft in one launch.
// With ssc_soma (a spiny stellate layer whose cells have one dendrite),
// ssc_cycle runs in the same launch (the step that follows the tuft's).
void launch_fused_tuft(const FusedArea& F, const uint8_t* axns, const SliceRec* slices, const DevLayer& L,
                       uint32_t layer, uint32_t t, AreaCtl* ctl, cudaStream_t s, bool ssc_soma = false,
                       int64_t host_cycle = -1);   // >= 0: the cycle number, for a launch that may run ahead of
                                                   // the area's counter
// Recomputes AreaCtl::tuft_status for the fused tufts of a layer (after its
// synapse sources or flags were written by the caller).
void launch_verify_tufts(const FusedArea& F, const DevLayer& L, uint32_t layer, AreaCtl* ctl, cudaStream_t s);
void launch_compile_tuft(const FusedArea& F, const DevLayer& L, uint32_t layer, uint32_t t, AreaCtl* ctl,
                         cudaStream_t s);

// Batched form: launches over several tufts (of one area or several).
struct FusedJob {
    const FusedArea* F;
    const DevLayer* L;
    const uint8_t* axns;
    const SliceRec* slices;
    AreaCtl* ctl;
    uint32_t layer, t;   // the tuft: data layer index and tuft index
    bool ssc_soma;       // ssc_cycle folded in (see launch_fused_tuft)
};
struct FusedBatch {
    bool ok = false;             // every job is tiled and the ring fits: batched launches serve them all
    bool tuft = false;           // pyramidal layer
    std::vector<void*> params;   // host parameter blocks, one launch each (up to 80 jobs of one
    std::vector<uint32_t> grids; // stage geometry per launch)
    std::vector<uint32_t> smems;
    uint32_t n_jobs = 0, n_tiles = 0;
};
// Launch shape of a batched tuft step, as the autotuner sets it: the ring's
// most stages (0: up to 4, fewest CTAs per SM lost) and the resident CTAs per
// SM of the persistent grid (0: as many as fit).
struct BatchShape {
    uint32_t max_stages = 0;
    uint32_t ctas_per_sm = 0;
};
// Plans the launches (B.ok false when some job cannot share them; the caller
// then launches each job's own form).
int prepare_fused_batch(FusedBatch& B, const std::vector<FusedJob>& jobs, const BatchShape& shape = {});
void launch_fused_batch(const FusedBatch& B, cudaStream_t s);
// Ring stages of one planned launch (an entry of FusedBatch::params).
uint32_t fused_batch_stages(const void* params);
void free_fused_batch(FusedBatch& B);

}  // namespace bm
