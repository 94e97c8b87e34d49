/*
 * bm_oracle.h -- CPU oracle for the bismit cortical cycle (TEST INFRASTRUCTURE).
 *
 * This is the checker, never the product: only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it. It restates bismit's OpenCL kernels
 * (cl/bismit.cl, cl/syns.cl, cl/control.cl) and the host stage order of
 * CorticalArea::cycle (src/cortex/cortical_area.rs:716-789) in plain C, on a
 * host copy of an area's state slab laid out by the resolved plan
 * (bm_area_plan in include/bismit_b200.h).
 *
 * The restatement is pinned against the reference's own kernel source compiled
 * for the CPU (oracle/ref/) and against the golden fixtures in tests/golden/.
 */
#ifndef BM_ORACLE_H
#define BM_ORACLE_H

#include <stdint.h>
#include "../include/bismit_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-launch random value: the same counter-based stream as bm_rnd. */
int32_t bmo_rnd(uint64_t seed, uint32_t area_id, uint32_t layer_id, uint32_t role,
                uint32_t tft_id, uint64_t cycle);

/* Writes bytes [off, off + len) of a frame of input `input` where intake puts
 * them: a source with a running filter chain into the chain's first buffer,
 * the rest into the input's axons. */
int bmo_intake(const bm_area_plan* plan, uint8_t* slab, uint32_t input, uint32_t off, const uint8_t* data,
               uint32_t len);

/* Runs n_cycles cycles on `slab` (plan->slab_bytes bytes). Before cycle k the
 * frame frames + k*frame_len (if frames != NULL) is written to input 0.
 * Cycle numbers start at start_cycle. n_threads <= 1 runs single-threaded. */
int bmo_run(const bm_area_plan* plan, uint8_t* slab, const uint8_t* frames, uint64_t frame_len,
            uint32_t n_cycles, uint64_t start_cycle, int n_threads);

/* Grows the synapses of every data layer (sources and strengths) exactly as the
 * library's growth kernel does (restatement of Synapses::grow(true),
 * src/cortex/synapses.rs:454-501, with the seeded per-dendrite stream). */
int bmo_grow(const bm_area_plan* plan, uint8_t* slab, uint64_t seed, uint32_t init_flags);

/* Hex offset list of gen_syn_offs (src/map/syn_src.rs:47-149); returns the
 * count written (<= cap) or -1 on error. */
int bmo_gen_syn_offs(int radius, uint32_t v_scale, uint32_t u_scale, int8_t* v_out,
                     int8_t* u_out, int cap);

/* Axon index pair of test_axn_idxs_scl / test_axn_idxs_vec4 (cl/tests.cl:15-85)
 * for one (slice, v, u, v_ofs, u_ofs): scalar and vec4 index formulas. */
uint32_t bmo_axn_idx_scl(const bm_area_plan* plan, uint8_t slc, uint32_t v, int8_t v_ofs,
                         uint32_t u, int8_t u_ofs, int* safe);
uint32_t bmo_axn_idx_vec4(const bm_area_plan* plan, uint8_t slc, int32_t v, int8_t v_ofs,
                          int32_t u, int8_t u_ofs, int* safe);

/* Input encoders (src/encode/), restated for checking the device encoders. */
void bmo_encode_image(const uint8_t* source, uint32_t x_size, uint32_t y_size, float scale_factor,
                      uint8_t* target, uint32_t v_size, uint32_t u_size);
int bmo_hex_mold(int radius, uint32_t src_v, uint32_t src_u, uint8_t* frame, uint32_t v_size, uint32_t u_size);
int bmo_encode_scalar(float val, float lo, float hi, uint64_t seed, uint32_t frame_idx, uint8_t* frame,
                      uint32_t v_size, uint32_t u_size);
int bmo_encode_scalar_glyph(float val, float lo, float hi, uint8_t* frame, uint32_t v_size, uint32_t u_size);
int bmo_sdr_waypoints(float lo, float hi, float way_span, uint32_t v_size, uint32_t u_size, uint64_t seed,
                      uint32_t* ways);
int bmo_sdr_encode(float val, float lo, float hi, float way_span, uint32_t way_count, const uint32_t* ways,
                   uint8_t* frame, uint32_t len);

#ifdef __cplusplus
}
#endif

#endif
