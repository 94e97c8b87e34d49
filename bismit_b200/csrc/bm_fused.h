// bm_fused.h -- the fused stage kernels: per-area preparation and launchers.
#pragma once
#include <string>

#include "bm_dev.cuh"

namespace bm {

struct FusedArea {
    int sms = 148;
    bool tuft_ok[BM_MAX_LAYERS][BM_MAX_TUFTS] = {};
    uint32_t slc0[BM_MAX_LAYERS][BM_MAX_TUFTS] = {};
    uint32_t nrec[BM_MAX_LAYERS][BM_MAX_TUFTS] = {};
};

// Decides, per tuft, whether the fused kernel applies (syns_per_den a power of
// two in 16..512, dens_per_tft a power of two, 16-byte aligned ranges). Tufts
// that do not qualify run the plain per-stage kernels.
int prepare_fused(FusedArea& F, const bm_area_plan& P, std::string* err);
void free_fused(FusedArea& F);
// Synapse flags + synapse cycle + dendrite cycle (+ tuft cycle for pyramidal
// layers) of one tuft in one launch.
void launch_fused_tuft(const FusedArea& F, const uint8_t* axns, const SliceRec* slices, const DevLayer& L,
                       uint32_t layer, uint32_t t, const AreaCtl* ctl, cudaStream_t s);

}  // namespace bm
