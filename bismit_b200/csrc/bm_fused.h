// bm_fused.h -- the fused stage kernels: per-area preparation and launchers.
#pragma once
#include <string>

#include "bm_dev.cuh"

namespace bm {

struct FusedArea {
    bool layer_ok[BM_MAX_LAYERS] = {};
};

// Decides, per data layer, whether the fused kernels apply to its scheme and
// buffer alignment. Returns BM_OK (layers that do not qualify use the plain form).
int prepare_fused(FusedArea& F, const bm_area_plan& P, const DevLayer* dl, uint8_t* slab, cudaStream_t s,
                  std::string* err);
void free_fused(FusedArea& F);
// Synapse sources of a layer were overwritten by the caller.
void mark_sources_dirty(FusedArea& F, uint32_t layer);
// Synapse flags + synapse cycle + dendrite cycle (+ tuft cycle for pyramidal
// layers) of one tuft in one launch.
void launch_fused_tuft(const FusedArea& F, const uint8_t* axns, const SliceRec* slices, const DevLayer& L,
                       uint32_t layer, uint32_t t, const AreaCtl* ctl, cudaStream_t s);

}  // namespace bm
