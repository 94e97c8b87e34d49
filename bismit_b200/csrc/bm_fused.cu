// bm_fused.cu -- fused stage kernels.
#include "bm_fused.h"

namespace bm {

int prepare_fused(FusedArea& F, const bm_area_plan& P, const DevLayer* dl, uint8_t* slab, cudaStream_t s,
                  std::string* err) {
    (void)P; (void)dl; (void)slab; (void)s; (void)err;
    for (int i = 0; i < BM_MAX_LAYERS; i++) F.layer_ok[i] = false;
    return BM_OK;
}
void free_fused(FusedArea& F) { (void)F; }
void mark_sources_dirty(FusedArea& F, uint32_t layer) { if (layer < BM_MAX_LAYERS) F.layer_ok[layer] = false; }
void launch_fused_tuft(const FusedArea&, const uint8_t*, const SliceRec*, const DevLayer&, uint32_t, uint32_t,
                       const AreaCtl*, cudaStream_t) {}

}  // namespace bm
