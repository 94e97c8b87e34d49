// bm_layout.h -- scheme resolution (bm_area_desc -> bm_area_plan) and growth specs.
#pragma once
#include <cstdarg>
#include <cstdint>
#include <string>
#include <vector>

#include "bm_dev.cuh"

namespace bm {

// One distinct source slice of a tuft with its offset pool.
struct GrowSrc {
    uint8_t slc = 0;
    uint8_t nonspatial = 0;
    int32_t rv = 0, ru = 0;
    std::vector<int8_t> offs_v, offs_u;
};

// Growth description of one tuft of one data layer.
struct TuftGrowSpec {
    uint32_t data_layer = 0, tft = 0;
    uint64_t key = 0;
    uint32_t n_pool = 0;
    uint8_t pool[BM_MAX_SRC_SLICES] = {};
    uint8_t pool_src[BM_MAX_SRC_SLICES] = {};
    std::vector<GrowSrc> srcs;
    bool saturated = false;
};

// Resolves the scheme; fills *grow with one spec per (data layer, tuft).
// Returns BM_OK or BM_ERR_INVALID with *err set.
int resolve_area(const bm_area_desc* D, uint64_t seed, bm_area_plan* P, std::vector<TuftGrowSpec>* grow,
                 std::string* err);

// Largest |v| and |u| offset in gen_syn_offs(reach, [vs, us]); false if the
// pool cannot be generated.
bool offset_extent(int reach, uint32_t vs, uint32_t us, int* rv, int* ru);

// Key of the per-launch random stream for (area, layer, role, tuft).
uint64_t rnd_key(uint64_t seed, uint32_t area, uint32_t layer, uint32_t role, uint32_t tft);
// The activity smoother's group centers for a host layer of v_size x u_size
// and group side r: six lattices, lattice k in out[off[k] .. off[k + 1]),
// each center packed as (v << 16) | (u & 0xFFFF) in 16-bit two's complement.
void smoother_centers(int r, int v_size, int u_size, std::vector<int32_t>& out, uint32_t off[7]);

// Key of the growth stream of (area, layer, tuft).
uint64_t grow_key(uint64_t seed, uint32_t area, uint32_t layer, uint32_t tft);

}  // namespace bm
