/*
 * bismit_b200.h -- C ABI of the B200-native bismit cortical cycle.
 *
 * This is the drop-in boundary for bismit's per-area cortical cycle plus
 * learning. Every entry point returns an int status (BM_OK == 0). Nothing
 * panics or aborts across this boundary; the last error message of the
 * calling thread is available from bm_last_error().
 *
 * Ownership: the library owns all device memory. Callers pass host buffers
 * (plain pointers and byte counts) which are only read or written for the
 * duration of the call.
 *
 * Threading: each handle is affine to one thread at a time. Separate areas may
 * be driven from separate threads; each area issues work on its own CUDA
 * stream (or the stream set with bm_ctx_set_stream).
 *
 * Reference interfaces replaced (paths relative to the bismit repository):
 *   bm_ctx_create        -> Cortex::new / OpenCL context    src/cortex/cortex.rs:51-61
 *   bm_area_create       -> CorticalArea::new               src/cortex/cortical_area.rs:376-615
 *                           (AreaMap::new src/map/area_map.rs:25, SliceMap::new
 *                           src/map/slice_map.rs:26, Synapses::grow
 *                           src/cortex/synapses.rs:454-501)
 *   bm_area_cycle        -> CorticalArea::cycle             src/cortex/cortical_area.rs:716-789
 *   bm_area_write_input  -> AxonSpace::intake               src/cortex/axon_space.rs:509-588
 *   bm_area_read_output  -> AxonSpace::output               src/cortex/axon_space.rs:594-629
 *   bm_sampler_*         -> CorticalArea::sampler + TractReceiver
 *                                                           src/cortex/cortical_area.rs:809-880,1017-1284
 *                                                           src/subcortex/tract_channel.rs:400-548
 *   bm_area_read/write   -> the *Test traits' buffer
 *                           read/write/fill helpers         src/cortex/cortical_area.rs:1017,1375-1516
 *                                                           src/cortex/synapses.rs:536-709
 *   bm_area_get_plan     -> AreaMap::gen_build_options (the resolved slice
 *                           tables and buffer index spaces) src/map/area_map.rs:51-77
 *   bm_last_error        -> CmnError / CmnResult            src/cmn/error.rs
 */
#ifndef BISMIT_B200_H
#define BISMIT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status -- */
#define BM_OK               0
#define BM_ERR_INVALID      1   /* bad argument or scheme                      */
#define BM_ERR_OOM          2   /* device allocation failed                    */
#define BM_ERR_CUDA         3   /* a CUDA runtime call failed                  */
#define BM_ERR_TIMEOUT      4   /* a bounded wait gave up                      */
#define BM_ERR_UNSUPPORTED  5   /* scheme feature outside this path            */
#define BM_ERR_NO_DEVICE    6   /* no CUDA device / device index out of range  */

/* ------------------------------------------------------------- limits ---- */
#define BM_MAX_SLICES       256 /* u8 slice ids (src/map/slice_map.rs:212)     */
#define BM_MAX_LAYERS       16
#define BM_MAX_TUFTS        4
#define BM_MAX_SRC_LAYERS   8
#define BM_MAX_SRC_SLICES   32  /* source-slice pool per tuft (with prevalence) */
#define BM_MAX_CTRL         4
#define BM_MAX_IO           8
#define BM_MAX_FILTERS      4   /* filters in one input filter chain            */
#define BM_NAME_LEN         32

/* Input filters (FilterScheme names, src/map/scheme/filter.rs; kernels of
 * cl/filters.cl). */
#define BM_FILTER_RETINA    1   /* "retina", cl/filters.cl:34-100 */

/* ------------------------------------------------------- layer schemes --- */
/* Layer kinds (src/map/scheme/layer.rs, src/map/mod.rs CellClass). */
#define BM_LYR_AXONAL              0
#define BM_LYR_SPINY_STELLATE      1
#define BM_LYR_PYRAMIDAL           2
#define BM_LYR_CTRL_INHIB_BASKET   3   /* InhibitoryBasketSurround -> inhib_simple  */
#define BM_LYR_CTRL_PYR_OUTPUT     4   /* PyrOutputter -> pyr_output                */
#define BM_LYR_CTRL_INTRA_COLUMN   5   /* IntraColumnInhib -> inhib_intra_column    */
#define BM_LYR_CTRL_SMOOTHER       6   /* ActivitySmoother -> smooth_activity       */

/* Axon domains (src/map/axon_domain.rs). */
#define BM_DOM_LOCAL   0
#define BM_DOM_INPUT   1
#define BM_DOM_OUTPUT  2

/* Axon topologies (src/map/mod.rs AxonTopology). */
#define BM_TOPO_SPATIAL     0
#define BM_TOPO_NONSPATIAL  1
#define BM_TOPO_NONE        2

/* Dendrite classes/kinds (src/map/mod.rs DendriteClass/DendriteKind). */
#define BM_DEN_BASAL     0
#define BM_DEN_APICAL    1
#define BM_DEN_PROXIMAL  0
#define BM_DEN_DISTAL    1

/* Layer tag bits, the high word of bismit's LayerTags (src/map/layer_tags.rs:121-150). */
#define BM_TAG_PRIMARY   (1ull << 32)
#define BM_TAG_SPATIAL   (1ull << 36)
#define BM_TAG_TEMPORAL  (1ull << 37)
#define BM_TAG_FOCUS     (1ull << 38)
#define BM_TAG_MOTOR     (1ull << 39)
#define BM_TAG_INPUT     (1ull << 48)
#define BM_TAG_OUTPUT    (1ull << 49)
#define BM_TAG_UNUSED    (1ull << 47)
#define BM_TAG_PSAL      (BM_TAG_PRIMARY | BM_TAG_SPATIAL)
#define BM_TAG_PTAL      (BM_TAG_PRIMARY | BM_TAG_TEMPORAL)

/* CorticalAreaSettings switches (src/cortex/cortical_area.rs:253-338). */
#define BM_SET_BYPASS_INHIB      (1u << 0)
#define BM_SET_BYPASS_FILTERS    (1u << 1)
#define BM_SET_DISABLE_PYRS      (1u << 2)
#define BM_SET_DISABLE_SSCS      (1u << 3)
#define BM_SET_DISABLE_MCOLS     (1u << 4)
#define BM_SET_DISABLE_REGROWTH  (1u << 5)
#define BM_SET_DISABLE_LEARNING  (1u << 6)

/* Growth options (bm_area_desc.init_flags). */
#define BM_INIT_STRENGTH_ZERO     (1u << 0)  /* strengths start at 0 (else the
                                                 SynSrcSlices::gen_src intensity x
                                                 U[-3,3] rule, src/map/syn_src.rs:448-490) */
#define BM_INIT_NO_UNIQUE         (1u << 1)  /* skip per-dendrite source uniqueness
                                                 (SynSrcIdxCache, src/map/syn_src.rs:159-211) */

/* Execution path (bm_area_desc.exec_path). */
#define BM_PATH_FUSED   0   /* fused stage kernels where the scheme allows (default) */
#define BM_PATH_PLAIN   1   /* one kernel per reference stage                         */

typedef struct bm_src_layer_desc {
    int32_t  layer_idx;    /* index into bm_area_desc.layers               */
    int32_t  syn_reach;    /* TuftSourceLayer::syn_reach (i8 range)          */
    uint32_t prevalence;   /* TuftSourceLayer::prevalence (>= 1)             */
} bm_src_layer_desc;

typedef struct bm_tuft_desc {
    uint32_t den_class;          /* BM_DEN_BASAL / BM_DEN_APICAL            */
    uint32_t den_kind;           /* BM_DEN_PROXIMAL / BM_DEN_DISTAL         */
    uint32_t dens_per_tft;
    uint32_t syns_per_den;
    uint32_t max_active_dens_l2;
    int64_t  thresh_init;        /* < 0: DENDRITE_DEFAULT_INITIAL_THRESHOLD (0) */
    uint32_t n_src;
    bm_src_layer_desc src[BM_MAX_SRC_LAYERS];
} bm_tuft_desc;

/* One source feeding an axonal input layer: the dims of the source layer the
 * thalamic tract delivers (LayerInfo::new, src/map/layer_info.rs:142-215),
 * and the filter chain its frames pass through on intake: the chain an
 * AreaScheme::filter_chain entry (src/map/scheme/area.rs:70-85) attaches to
 * the one source whose input signature it names
 * (LayerMap::src_layer_info_by_sig, src/map/layer_map.rs:242-261). */
typedef struct bm_input_src_desc {
    uint32_t v_size, u_size, depth;
    uint32_t axon_topology;
    uint32_t n_filters;                /* 0: frames written straight to the axons */
    uint32_t filters[BM_MAX_FILTERS];  /* BM_FILTER_*, first applied first        */
} bm_input_src_desc;

typedef struct bm_layer_desc {
    char     name[BM_NAME_LEN];
    uint64_t tags;               /* BM_TAG_* bits                              */
    uint32_t kind;               /* BM_LYR_*                                   */
    int32_t  depth;              /* < 0: unset (0 for local/output layers)     */
    uint32_t axon_topology;      /* BM_TOPO_*                                  */
    uint32_t axon_domain;        /* BM_DOM_*                                   */
    /* Axonal input layers: the sources (one slice range per source). */
    uint32_t n_input_srcs;
    bm_input_src_desc input_srcs[BM_MAX_IO];
    /* Control layers. */
    int32_t  host_layer_idx;
    uint32_t field_radius;
    uint32_t exe_order;
    /* Cellular layers. */
    uint32_t n_tufts;
    bm_tuft_desc tufts[BM_MAX_TUFTS];
} bm_layer_desc;

typedef struct bm_area_desc {
    uint32_t area_id;
    uint32_t v_size, u_size;     /* area column grid                          */
    uint32_t n_layers;
    bm_layer_desc layers[BM_MAX_LAYERS];
    uint32_t settings;           /* BM_SET_*                                   */
    uint32_t init_flags;         /* BM_INIT_*                                  */
    uint32_t exec_path;          /* BM_PATH_*                                  */
} bm_area_desc;

/* ------------------------------------------------------- resolved plan --- */
/* The resolved index spaces of an area: slice tables, per-layer buffer
 * offsets within the area's state slab, tuft index ranges. Used by callers
 * that address raw buffers (tests, samplers, snapshots) and by the oracle.    */

/* Buffer kinds within a layer (mirrors SamplerKind, src/cortex/cortical_area.rs:61-90). */
#define BM_BUF_SYN_STATES               0
#define BM_BUF_SYN_STRENGTHS            1
#define BM_BUF_SYN_SRC_SLC_IDS          2
#define BM_BUF_SYN_SRC_COL_V_OFFS       3
#define BM_BUF_SYN_SRC_COL_U_OFFS       4
#define BM_BUF_SYN_FLAG_SETS            5
#define BM_BUF_DEN_STATES_RAW           6
#define BM_BUF_DEN_STATES               7
#define BM_BUF_DEN_ENERGIES             8
#define BM_BUF_DEN_ACTIVITIES           9
#define BM_BUF_DEN_THRESHOLDS           10
#define BM_BUF_TFT_PREV_BEST_DEN_IDS    11
#define BM_BUF_TFT_PREV_BEST_DEN_STATES_RAW 12
#define BM_BUF_TFT_PREV_BEST_DEN_STATES 13
#define BM_BUF_TFT_PREV_STATES          14
#define BM_BUF_TFT_BEST_DEN_IDS         15
#define BM_BUF_TFT_BEST_DEN_STATES_RAW  16
#define BM_BUF_TFT_BEST_DEN_STATES      17
#define BM_BUF_TFT_STATES               18
#define BM_BUF_CEL_ENERGIES             19
#define BM_BUF_CEL_ACTIVITIES           20
#define BM_BUF_CEL_STATES               21   /* pyramidal soma                     */
#define BM_BUF_CEL_FLAG_SETS            22   /* pyramidal cell flags               */
#define BM_BUF_DEN_SRC_KEY0             23   /* per dendrite, regrowth on only: key 0
                                                 held in the dendrite's source set
                                                 (SynSrcIdxCache, src/map/syn_src.rs:159-211) */
#define BM_BUF_COUNT                    24
#define BM_BUF_AXON_STATES              64   /* area axon space (layer ignored)    */

typedef struct bm_tuft_plan {
    uint32_t tft_id, den_class, den_kind;
    uint32_t dens_per_tft, syns_per_den, syns_per_tft;
    uint32_t max_active_dens_l2;
    uint32_t den_threshold;
    uint64_t syn_idz;      /* first synapse of the tuft (layer-relative)      */
    uint64_t den_idz;      /* first dendrite of the tuft (layer-relative)     */
    uint64_t cel_idz;      /* tft_id * cells (cell-tuft index base)           */
    uint32_t n_src;        /* pool with prevalence repeats                    */
    uint8_t  src_slc_ids[BM_MAX_SRC_SLICES];
    int8_t   src_reaches[BM_MAX_SRC_SLICES];
    uint32_t n_src_uniq;   /* distinct (slice, reach) pairs                  */
    uint8_t  src_uniq_slc_ids[BM_MAX_SRC_SLICES];
    int8_t   src_uniq_reaches[BM_MAX_SRC_SLICES];
} bm_tuft_plan;

typedef struct bm_ctrl_plan {
    uint32_t kind;          /* BM_LYR_CTRL_*                                  */
    uint32_t exe_order;
    uint32_t field_radius;
    uint32_t layer_id;
} bm_ctrl_plan;

typedef struct bm_layer_plan {
    uint32_t layer_id;      /* index in the area's layer list                */
    uint32_t kind;          /* BM_LYR_SPINY_STELLATE / BM_LYR_PYRAMIDAL        */
    uint64_t tags;
    uint32_t depth;
    uint32_t base_axn_slc;
    uint32_t axn_idz;
    uint32_t v_size, u_size;
    uint32_t cells;
    uint32_t n_tufts;
    bm_tuft_plan tufts[BM_MAX_TUFTS];
    uint64_t n_syns, n_dens, n_celtfts;
    uint32_t enabled_tft_flags;  /* pyramidal: DEN_*_FLAG bits               */
    uint32_t bsl_prx_tft_id, bsl_dst_tft_id, apc_dst_tft_id;
    uint32_t n_ctrl;
    bm_ctrl_plan ctrl[BM_MAX_CTRL];   /* post-cycle controls, (host, exe_order) order */
    uint64_t buf_off[BM_BUF_COUNT];   /* byte offset in the state slab, or UINT64_MAX */
    uint64_t buf_len[BM_BUF_COUNT];   /* bytes                                         */
} bm_layer_plan;

typedef struct bm_io_plan {
    uint32_t layer_idx;     /* scheme layer index                             */
    uint32_t axn_idz;       /* first axon                                     */
    uint32_t len;           /* axons                                          */
} bm_io_plan;

/* One input filter chain (AxonSpace::new, src/cortex/axon_space.rs:338-412):
 * filter k reads its input buffer (depth x v_size x u_size bytes) and writes
 * the next filter's, the last one the target axon slices. Frames for the
 * source land in the first buffer; the chain runs at the head of every cycle
 * unless BM_SET_BYPASS_FILTERS is set (AxonSpace::intake, :510-525). */
typedef struct bm_filter_chain_plan {
    uint32_t input;          /* index into bm_area_plan.inputs                */
    uint32_t frame_off;      /* the source's first byte within that input      */
    uint32_t tar_slc;        /* first target axon slice (tar_slc_range.start)  */
    uint32_t depth, v_size, u_size;
    uint32_t n_filters;
    uint32_t filters[BM_MAX_FILTERS];
    uint64_t buf_off[BM_MAX_FILTERS];  /* each filter's input buffer in the slab */
} bm_filter_chain_plan;

typedef struct bm_area_plan {
    uint32_t area_id;
    uint32_t v_size, u_size;
    uint32_t settings;
    uint32_t n_slices;
    uint32_t slc_axn_idz[BM_MAX_SLICES];
    uint32_t slc_v_size[BM_MAX_SLICES];
    uint32_t slc_u_size[BM_MAX_SLICES];
    uint32_t slc_v_scale[BM_MAX_SLICES];
    uint32_t slc_u_scale[BM_MAX_SLICES];
    uint32_t slc_v_mid[BM_MAX_SLICES];
    uint32_t slc_u_mid[BM_MAX_SLICES];
    uint32_t slc_layer[BM_MAX_SLICES];   /* owning scheme layer               */
    uint32_t n_axons;
    uint64_t axon_off;                   /* axon space offset in the slab     */
    uint32_t n_inputs;
    bm_io_plan inputs[BM_MAX_IO];
    uint32_t n_outputs;
    bm_io_plan outputs[BM_MAX_IO];
    uint32_t n_layers;                   /* data (cellular) layers            */
    bm_layer_plan layers[BM_MAX_LAYERS];
    uint32_t n_cycle_order;              /* data layers in role order         */
    uint32_t cycle_order[BM_MAX_LAYERS]; /* indices into layers[]            */
    uint64_t slab_bytes;
    uint64_t n_syns_total;
    uint64_t rnd_seed;                   /* per-launch random stream key      */
    uint32_t n_filter_chains;
    bm_filter_chain_plan filter_chains[BM_MAX_IO];
} bm_area_plan;

/* ------------------------------------------------------------ handles ---- */
typedef struct bm_ctx_s*  bm_ctx;
typedef struct bm_area_s* bm_area;

/* Thread-local message for the last failing call ("" if none). */
const char* bm_last_error(void);

/* Version string of this library. */
const char* bm_version(void);

/* Creates a context on CUDA device `device` (Cortex::new, src/cortex/cortex.rs:51-61). */
int bm_ctx_create(int device, uint32_t flags, bm_ctx* out);
/* Releases the caller's handle. Areas, batches, servers and writers made on
 * the context hold it too, so it may be destroyed before them (as a garbage
 * collector may order it): it is freed with the last of them. The handle
 * must not be used after this call. */
int bm_ctx_destroy(bm_ctx ctx);
/* Issues all subsequent work of areas created from ctx on `stream` (a
 * cudaStream_t passed as void*; NULL is the CUDA legacy default stream).
 * bm_ctx_use_own_stream returns to the library's own non-blocking stream. */
int bm_ctx_set_stream(bm_ctx ctx, void* stream);
int bm_ctx_use_own_stream(bm_ctx ctx);
/* Blocks until all work issued through ctx has finished. */
int bm_ctx_synchronize(bm_ctx ctx);

/* Builds an area from a scheme, allocates its state and grows its synapses from
 * the seeded stream `seed` (CorticalArea::new, src/cortex/cortical_area.rs:376). */
int bm_area_create(bm_ctx ctx, const bm_area_desc* desc, uint64_t seed, bm_area* out);
int bm_area_destroy(bm_area area);

/* Copies the resolved plan (slice tables, buffer offsets) to *out. */
int bm_area_get_plan(bm_area area, bm_area_plan* out);

/* Resolves a scheme into its plan without creating an area or touching a
 * device (the AreaMap::new half of CorticalArea::new). */
int bm_plan_resolve(const bm_area_desc* desc, uint64_t seed, bm_area_plan* out);

/* Writes one thalamic frame into the axon range of input layer `input_idx`
 * (index into plan.inputs); len must equal that range (AxonSpace::intake,
 * src/cortex/axon_space.rs:509-588). The copy is ordered before the next cycle.
 * The frame's bytes are read during the call only, pinned or pageable: the
 * caller may reuse its buffer as soon as the call returns. The upload runs
 * beside the cycles already enqueued. */
int bm_area_write_input(bm_area area, uint32_t input_idx, const uint8_t* frame, size_t len);

/* Same, from device memory (a frame already resident in HBM). */
int bm_area_write_input_device(bm_area area, uint32_t input_idx, const void* dev_frame, size_t len);

/* Runs n_cycles full cycles: intake is whatever was written before, then the
 * spatial layers, their learning, the temporal layers with control layers and
 * learning (CorticalArea::cycle, src/cortex/cortical_area.rs:716-789). Work is
 * enqueued asynchronously on the area's stream. */
int bm_area_cycle(bm_area area, uint32_t n_cycles);

/* Like bm_area_cycle with one fresh input frame per cycle taken from a device
 * array of n_cycles frames of `frame_len` bytes each (input 0). */
int bm_area_cycle_frames_device(bm_area area, const void* dev_frames, size_t frame_len,
                                uint32_t n_cycles);

/* Reads the axons of output layer `output_idx` (AxonSpace::output,
 * src/cortex/axon_space.rs:594-629). Synchronous. */
int bm_area_read_output(bm_area area, uint32_t output_idx, uint8_t* dst, size_t len);

/* Reads/writes `len` bytes at byte `offset` of buffer `buf_kind` of data layer
 * `layer` (plan index; ignored for BM_BUF_AXON_STATES). Synchronous. */
int bm_area_read(bm_area area, uint32_t buf_kind, uint32_t layer, uint64_t offset,
                 void* dst, uint64_t len);
int bm_area_write(bm_area area, uint32_t buf_kind, uint32_t layer, uint64_t offset,
                  const void* src, uint64_t len);

/* Whole-state snapshot and restore (the slab, plan.slab_bytes) plus the cycle counter. */
int bm_area_read_slab(bm_area area, void* dst, uint64_t len);
int bm_area_write_slab(bm_area area, const void* src, uint64_t len);
int bm_area_get_cycle(bm_area area, uint64_t* out);
int bm_area_set_cycle(bm_area area, uint64_t cycle);

/* ------------------------------------------------------------- samplers -- */
/* Per-cycle readback of one buffer of an area through a one-frame channel:
 * CorticalArea::sampler (src/cortex/cortical_area.rs:1017-1284,
 * SamplerBufferKind::Single) with the tract channel of
 * src/subcortex/tract_channel.rs:400-488. After every cycle of the area
 * (bm_area_cycle, bm_area_cycle_frames_device, bm_batch_cycle,
 * bm_batch_cycle_frames_device) the sampler sends a frame if the receiver has
 * taken the last one; if not, the new frame is skipped, or with backpressure
 * the cycling call waits until the receiver takes it (another thread calls
 * bm_sampler_recv). A frame is an asynchronous copy after the cycle's
 * kernels; bm_sampler_recv waits for it. Samplers belong to their area and
 * are destroyed with it. */
typedef struct bm_sampler_s* bm_sampler;
#define BM_ALL_LAYERS 0xFFFFFFFFu   /* with BM_BUF_AXON_STATES: every axon of the area */

/* kind: a BM_BUF_* buffer of data layer `layer` (the whole buffer, every
 * tuft: SomaStates .. SynFlagSets), or BM_BUF_AXON_STATES for the axons of
 * layer `layer` (its slices) or of the whole area (BM_ALL_LAYERS):
 * SamplerKind::Axons, src/cortex/cortical_area.rs:61-90. */
int bm_sampler_create(bm_area area, uint32_t kind, uint32_t layer, int backpressure, bm_sampler* out);
int bm_sampler_destroy(bm_sampler sampler);
int bm_sampler_len(bm_sampler sampler, uint64_t* len);
/* TractSender/TractReceiver::set_backpressure (tract_channel.rs:496-503). */
int bm_sampler_set_backpressure(bm_sampler sampler, int on, int* prior);
/* Bounds the waits of bm_sampler_recv and of a backpressured cycle (ms; 0,
 * the default, waits forever as the reference does); a wait that runs out
 * returns BM_ERR_TIMEOUT. */
int bm_sampler_set_timeout(bm_sampler sampler, uint32_t ms);
/* TractReceiver::recv (tract_channel.rs:438-488): copies the unread frame
 * (`len` = bm_sampler_len) to dst and sets *got = 1 and *cycle to the cycle
 * whose end state it holds; with no unread frame, waits for the next one if
 * wait_for_frame, else sets *got = 0. */
int bm_sampler_recv(bm_sampler sampler, int wait_for_frame, void* dst, uint64_t len, uint64_t* cycle,
                    int* got);
/* Frames sent, and frames skipped because one was unread. */
int bm_sampler_stats(bm_sampler sampler, uint64_t* sent, uint64_t* skipped);

/* Device pointer of the state slab (for callers that move data with their own
 * copies on the same device). A caller that writes synapse sources or flags
 * through it must call bm_area_sources_changed for that layer before the next
 * cycle; one that reads or writes axons (its own tract copies, say) with work
 * queued on the area's stream must call bm_area_axons_touched after queueing
 * it. */
int bm_area_slab_ptr(bm_area area, void** out);
/* The caller queued reads or writes of the area's axons on its stream
 * (through bm_area_slab_ptr): the next cycle's front steps, which otherwise
 * wait only for the previous cycle's steps they touch the buffers of, wait for
 * the stream's current position. The area's own intakes and reads
 * (bm_area_write_*, bm_area_read*, bm_area_deliver_tract, samplers) need no
 * call. */
int bm_area_axons_touched(bm_area area);
/* Steps of the area's cycle that run on its side stream, beside the chain of
 * steps they do not touch (tuft steps that depend on nothing earlier in the
 * cycle, e.g. pyramidal distal tufts). Caller-written source slice ids
 * outside a tuft's pool keep that tuft's steps in the chain. */
int bm_area_side_steps(bm_area area, uint32_t* n);
/* Leading steps of the area's cycle that run on its front stream (0: none
 * this cycle): the spatial layers' fused tuft and inhibition launches, with
 * the frame intake. Each waits only for the steps of the previous cycle it
 * touches the buffers of, so one cycle's spatial chain runs beside the
 * previous cycle's pyramidal steps; they take the cycle number from the host.
 * Not used while profiling, or while a sampler reads a buffer they write. */
int bm_area_front_steps(bm_area area, uint32_t* n);
int bm_area_sources_changed(bm_area area, uint32_t layer);

/* One tract's delivery between two areas of a cortex cycled one area after
 * another, as bismit's Cortex::cycle does (src/cortex/cortex.rs:99-119): the
 * current axons of output `src_output` of `src` -- what its latest cycle
 * wrote, read by CorticalArea::output into the thalamic tract,
 * src/cortex/axon_space.rs:594-629 -- into input `dst_input` of `dst` at axon
 * `dst_offset`, landing where AxonSpace::intake puts a tract frame
 * (src/cortex/axon_space.rs:509-588; a filtered source's bytes into its
 * chain's first buffer). Enqueued on dst's stream after the work already
 * queued for src; src's next cycle follows the copy. A batch with tracts
 * (bm_batch_connect) instead delivers every tract at the head of each cycle,
 * from the previous cycle. */
int bm_area_deliver_tract(bm_area src, uint32_t src_output, bm_area dst, uint32_t dst_input, uint64_t dst_offset);

/* Sticky device-side error bits of the area (bit 0: a bounded wait inside a
 * kernel gave up). Synchronous; returns BM_ERR_TIMEOUT when any bit is set.
 * No reference counterpart (bismit panics on errors, src/cortex/cortex.rs:111).
 * A cycle that ends with error bits set also copies them to host memory the
 * library reads without synchronising: the area's (or a batch holding it)
 * next cycling call then returns BM_ERR_TIMEOUT without enqueueing anything,
 * until bm_area_clear_errors. */
int bm_area_device_errors(bm_area area, uint32_t* bits);
/* Clears the area's device error bits (after the caller restored a state it
 * trusts, e.g. with bm_area_write_slab). Synchronous. */
int bm_area_clear_errors(bm_area area);
/* Limit, in microseconds, of every bounded wait inside the area's tuft
 * kernels (0: the default, 2 s). A wait that runs out sets error bit 0, the
 * kernel lets its own copies land and returns. Synchronous. */
int bm_area_set_wait_limit(bm_area area, uint32_t us);
/* Fault injection for tests of the give-up path: in every tiled tuft launch
 * of the area (alone or batched), the copy lane of the block that takes the
 * tuft's first tile withholds the `stage`-th shared-memory stage it issues
 * from that tile on (counted from 1; 0 switches it off), so the consumers'
 * bounded wait for it runs out. Nothing faults: every wait stays bounded.
 * Synchronous. */
int bm_area_inject_stall(bm_area area, uint32_t stage);

/* How the fused path runs tuft `tuft` of data layer `layer` (no reference
 * counterpart: bismit runs one kernel per stage). For tests and profiling,
 * which form a workload exercises. All zero when the tuft takes the plain
 * per-stage or per-cell kernels. Synchronous. */
typedef struct bm_tuft_form {
    uint32_t fused;            /* the fused tuft kernel runs it                        */
    uint32_t tiled;            /* it gathers from a shared-memory axon footprint       */
    uint32_t consumer;         /* compile-time specialised consumer shape (1..7), 0 =
                                  the general one                                      */
    uint32_t sources_outside;  /* a source lies outside the footprint: checked gathers */
    uint32_t flags_foreign;    /* a flag byte has bits besides SYN_PREV_ACTIVE: flags
                                  stream through and keep those bits                   */
    uint32_t tile_w, tile_h;   /* cells per tile (tiled form)                          */
    uint32_t stages;           /* shared-memory ring stages                            */
    uint32_t grid;             /* persistent CTAs                                      */
    uint32_t smem;             /* dynamic shared memory per CTA, bytes                 */
    uint32_t footprint_tma;    /* 1: each tile's axon footprint arrives as one tensor
                                  box load (else the consumer warps stage it)          */
} bm_tuft_form;
int bm_area_tuft_form(bm_area area, uint32_t layer, uint32_t tuft, bm_tuft_form* out);

/* Per-kernel CUDA-event timing of subsequent cycles (0 = off). */
int bm_area_set_profiling(bm_area area, int on);
/* Per kernel kind: launch count and summed device milliseconds since the last
 * reset; names are static strings. n_max entries at most; *n_out = written. */
int bm_area_get_profile(bm_area area, uint32_t n_max, const char** names,
                        uint64_t* launches, double* ms, uint32_t* n_out);
int bm_area_reset_profile(bm_area area);

/* Number of kernel launches bm_area_cycle issues per cycle for this area. */
int bm_area_launches_per_cycle(bm_area area, uint32_t* out);

/* ------------------------------------------------------------- batches ---
 * A batch cycles several areas together, of uneven column-grid sizes and
 * possibly different layer maps. It schedules one sequence of stage steps
 * that contains every area's own step sequence in order, and runs each step
 * as one launch over all areas that have it; the whole cycle is captured once
 * as a CUDA graph and replayed. Every area keeps its own state; an area's bytes after a batched
 * cycle are the bytes it would have after bm_area_cycle alone (given the same
 * inputs). Replaces bismit's one-area-at-a-time loop
 * over areas in Cortex::cycle (src/cortex/cortex.rs:99-119), where every area
 * enqueues its own kernels.
 *
 * The areas stay owned by the caller and usable on their own (reads, writes,
 * bm_area_cycle); destroy the batch before any of its areas. */
typedef struct bm_batch_s* bm_batch;

int bm_batch_create(bm_ctx ctx, const bm_area* areas, uint32_t n_areas, bm_batch* out);
int bm_batch_destroy(bm_batch batch);

/* Graph capture and replay of the cycle (default on); off: the same launches
 * issued every cycle. */
int bm_batch_set_graph(bm_batch batch, int on);

/* n cycles of every area, inputs as last written to each area. */
int bm_batch_cycle(bm_batch batch, uint32_t n_cycles);

/* A tract: output `src_output` of area `src_area` (batch indices) feeds input
 * `dst_input` of area `dst_area` at axon offset `dst_offset` within that input
 * layer (an input layer fed by several source areas holds their slices one
 * after another). At the head of every batched cycle each tract copies its
 * source's output axons as they were at the end of the previous cycle, so all
 * areas of a cycle see the previous cycle's outputs. Replaces the thalamic
 * routing of bismit's Thalamus (src/subcortex/thalamus/thalamus.rs:97-112,
 * 193-238) between the areas of one cortex, whose tracts are read by
 * AxonSpace::intake (src/cortex/axon_space.rs:509-588). */
int bm_batch_connect(bm_batch batch, uint32_t src_area, uint32_t src_output, uint32_t dst_area,
                     uint32_t dst_input, uint64_t dst_offset);

/* Bytes of one cycle's frame block: every input of every area that no tract
 * feeds, packed in (area, input) order. */
int bm_batch_frame_bytes(bm_batch batch, uint64_t* out);

/* n cycles, each first copying its frame block (cycle k at dev_frames +
 * k * frame_bytes) into those inputs. */
int bm_batch_cycle_frames_device(bm_batch batch, const void* dev_frames, uint32_t n_cycles);

/* Kernel launches per batched cycle (all areas together). */
int bm_batch_launches_per_cycle(bm_batch batch, uint32_t* out);

/* Per-step CUDA-event timing of later cycles (the graph is bypassed while
 * on). bm_batch_get_profile reports, per scheduled step that ran: its step
 * kind (+1000 when it ran as one batched fused-tuft launch), layer, tuft or
 * control index, number of areas, launches and summed device milliseconds;
 * n_max entries at most, *n_out written. Arrays may be NULL. */
int bm_batch_set_profiling(bm_batch batch, int on);
int bm_batch_get_profile(bm_batch batch, uint32_t n_max, uint32_t* kinds, uint32_t* layers, uint32_t* idx,
                         uint32_t* n_areas, uint64_t* launches, double* ms, uint32_t* n_out);
int bm_batch_reset_profile(bm_batch batch);

/* OR of the areas' sticky device error bits; BM_ERR_TIMEOUT when any is set. */
int bm_batch_device_errors(bm_batch batch, uint32_t* bits);

/* Chooses, for each batched tuft step, the tile size (4K..128K synapses per
 * tile) and the footprint form (a tensor box load, or staged by the
 * consumers), then for those tiles the ring's depth (2..4 shared-memory
 * stages) and the resident CTAs per SM of the persistent grid, by timing
 * candidates on the batch itself (the buffers the trials write are saved and
 * restored, so the areas' state is unchanged). With a non-NULL cache_path,
 * choices already in that file are applied without timing and new ones are
 * added to it (one line per step: key, tile target, stages, CTAs per SM,
 * staged footprints; 0 = the default). *n_tuned (optional) = steps tuned.
 * Synchronous. */
int bm_batch_autotune(bm_batch batch, const char* cache_path, uint32_t* n_tuned);

/* One tuft's stage of a cycle -- synapse flags, synapse cycle, dendrite cycle,
 * and for pyramidal layers the tuft cycle -- on a state slab the CALLER owns,
 * without allocating any device memory. No counterpart in the reference: bismit
 * allocates every buffer when the area is built and has no such mode.
 *
 * For callers that must not allocate: a host whose device memory all comes
 * from its own pooling allocator (a foreign cudaMalloc would fail against its
 * reserve or escape its accounting), a real-time loop that cannot take
 * cudaMalloc's latency or cudaFree's implicit device synchronisation, or a
 * plugin handed pre-allocated buffers only. Such a caller resolves the plan
 * with bm_plan_resolve (host only), allocates plan->slab_bytes itself and
 * passes the slab here with the current device set.
 *
 * `slab` is the device state laid out by `plan` (inputs and outputs both
 * live there: axons, synapse sources, strengths and flags are read; synapse
 * states and flags, dendrite states and activities and the tuft's cell-tuft
 * buffers are written). `cycle` is the cycle number the per-launch random
 * value is drawn for (bm_rnd). `dev_error_out`, if not NULL, is a device word
 * the call sets to its device error bits (bit 0: a bounded wait gave up).
 * Work is queued on `stream` (NULL: the default stream); the call does not
 * wait for it.
 *
 * Scratch: one library-held device array of about 8 MiB, reserved on every
 * device that loads the library until the process exits. It limits a call to
 * tufts of at most 4,194,304 synapses (cells * syns_per_tft); larger tufts
 * get BM_ERR_INVALID, and tufts outside the fused kernel's shapes
 * BM_ERR_UNSUPPORTED. The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress, which may load the module), and so does the
 * first call after the device's context was replaced (cudaDeviceReset); make
 * those calls before any stream capture. An error already pending in the
 * calling thread (cudaPeekAtLastError) is returned as BM_ERR_CUDA and left
 * pending. Every call shares the array and leaves its
 * contents behind; the call re-initialises what it reads, but calls whose work
 * overlaps on the GPU (different streams or threads, same device) race on
 * it and must be serialised by the caller. Calls no cudaMalloc or cudaFree. */
int bm_tuft_cycle_static(const bm_area_plan* plan, uint32_t layer, uint32_t tuft, void* slab,
                         uint64_t cycle, uint32_t* dev_error_out, void* stream);

/* ------------------------------------------------------------- serving ---
 * A continuous-batching server over cortex sessions (one area each, with
 * exactly one input layer). bm_server_open queues a session; it is admitted
 * when the device-memory budget has room for its whole state (computed from
 * its resolved plan before anything is allocated), in FIFO order, and stays
 * resident until closed and drained. Each bm_server_tick cycles every
 * resident session that has a pending frame exactly once, all in one batch
 * (rebuilt only when that set changes). Admitted sessions' areas are built
 * and grown by a thread the server owns, on a stream of their own, and join
 * the first tick after they are ready, so no tick waits for a set-up (or a
 * teardown, which that thread does too). A session whose area ends a cycle
 * with device error bits (a bounded wait gave up) is dropped with its queued
 * frames: the tick that finds it returns BM_ERR_TIMEOUT once, later ticks
 * run the other sessions, and reading its output returns BM_ERR_TIMEOUT.
 * No counterpart in the reference, which cycles a fixed set of areas
 * (Cortex::cycle, src/cortex/cortex.rs:99-119). */
typedef struct bm_server_s* bm_server;

typedef struct bm_server_stats {
    uint64_t ticks, frames, batch_rebuilds;
    double   syn_cycles;          /* synapse-cycles done                         */
    double   busy_s;              /* summed tick spans (queue to completion)     */
    double   rebuild_s, admit_s;  /* host time in batch rebuilds / admissions    */
    double   gpu_s;               /* device time of the ticks                    */
    double   span_s;              /* first tick start to last tick end           */
    double   p50_ms, p99_ms, mean_ms;  /* per-frame latency: completion minus the
                                     moment the frame was ready (submitted, or its
                                     session's previous frame done)              */
    uint64_t used_bytes, budget_bytes;
    uint32_t resident, waiting;
    uint32_t failed;              /* sessions dropped after a device error       */
    uint64_t rebuild_drains;      /* rebuilds that waited for the queued ticks
                                     (a staging block grew)                      */
    double   capture_s;           /* host time of the ticks that captured a
                                     batch's CUDA graph (a batch cycles by plain
                                     launches until its membership has held for
                                     8 ticks)                                    */
    double   tick_p99_ms, tick_max_ms; /* device time of a tick: 99th percentile
                                     and largest                                 */
    uint64_t tick_max_no;         /* the slowest tick: its number (0: the first),  */
    uint32_t tick_max_members;    /* its sessions, and BM_TICK_* bits of what the  */
    uint32_t tick_max_what;       /* call that queued it also did                  */
    double   tick_max_queue_ms;   /* host time queueing its work took              */
    uint32_t tick_max_builder;    /* BM_BUILDER_* kinds of the builder thread's
                                     operations between its queueing and its
                                     completion, and the longest one's host ms   */
    uint32_t pad0;
    double   tick_max_builder_ms;
} bm_server_stats;

/* bm_server_stats.tick_max_builder */
#define BM_BUILDER_BUILD          1u   /* a session's area built and grown      */
#define BM_BUILDER_BATCH          2u   /* a retired batch released               */
#define BM_BUILDER_DEVICE_BUFFER  4u   /* a retired gather table released        */
#define BM_BUILDER_AREA_FREE      8u   /* a retired session's area released      */
#define BM_BUILDER_OUTPUT_FREE   16u   /* a retired session's output buffer freed */

/* bm_server_stats.tick_max_what */
#define BM_TICK_FIRST   1u   /* the server's first tick                  */
#define BM_TICK_REBUILD 2u   /* a new batch for a new membership         */
#define BM_TICK_DRAIN   4u   /* the rebuild waited for the queued ticks  */
#define BM_TICK_CAPTURE 8u   /* the batch's CUDA graph was captured      */

/* mem_budget 0: 90 % of the device memory free at creation. */
int bm_server_create(bm_ctx ctx, uint64_t mem_budget, bm_server* out);
int bm_server_destroy(bm_server server);
/* Queues a session; BM_ERR_OOM if it could never fit the budget. */
int bm_server_open(bm_server server, const bm_area_desc* desc, uint64_t seed, uint32_t* session);
/* Appends n_frames input frames (copied). */
int bm_server_submit(bm_server server, uint32_t session, const uint8_t* frames, size_t frame_len,
                     uint32_t n_frames);
/* The session leaves once its submitted frames are cycled. */
int bm_server_close(bm_server server, uint32_t session);
/* Closes a session and discards its queued frames (frames already in a
 * queued tick still complete). */
int bm_server_cancel(bm_server server, uint32_t session);
/* Queues one tick (*n_cycled, optional: sessions in it) and completes the
 * previous one: ticks are pipelined two deep, so a session's output and
 * frame count reflect the tick before the latest. Returns at once with
 * *n_cycled 0 when no resident session has a frame (sessions may still be
 * being built). */
int bm_server_tick(bm_server server, uint32_t* n_cycled);
/* Completes every queued tick. */
int bm_server_drain(bm_server server);
/* Output 0 after the session's latest cycled frame; *frames_done (optional). */
int bm_server_read_output(bm_server server, uint32_t session, uint8_t* dst, size_t len, uint64_t* frames_done);
/* The session's area while it is resident (NULL while waiting). */
int bm_server_session_area(bm_server server, uint32_t session, bm_area* out);
int bm_server_get_stats(bm_server server, bm_server_stats* out);
int bm_server_reset_stats(bm_server server);

/* The per-launch random value the host would draw for (layer, role, tuft) at
 * `cycle` (replaces the SmallRng draws of src/cortex/dendrites.rs:198,
 * src/cortex/tufts.rs:312, src/cortex/spiny_stellates.rs:259,
 * src/cortex/iinn.rs:113). */
#define BM_RND_DEN_CYCLE   1
#define BM_RND_INHIB       2
#define BM_RND_SSC_MTP     3
#define BM_RND_TFT_DST_MTP 4
int32_t bm_rnd(uint64_t seed, uint32_t area_id, uint32_t layer_id, uint32_t role,
               uint32_t tft_id, uint64_t cycle);

/* ------------------------------------------------------------ encoders ---
 * Input encoders (src/encode/) as kernels writing frames in device memory on
 * the context's stream. The f32 arithmetic follows the reference's operation
 * by operation; its entropy-seeded random bytes and waypoint indices come
 * from a seeded stream here. Frames are `frame_stride` bytes apart. */

/* encode_2d_image (src/encode/mod.rs:66-93): n images of x_size x y_size
 * bytes (contiguous, device) resampled onto v_size x u_size hexagonal frames
 * (device). Cells whose pixel falls outside the image keep their bytes. */
int bm_encode_images(bm_ctx ctx, const uint8_t* images, uint32_t n, uint32_t x_size, uint32_t y_size,
                     float scale_factor, uint8_t* frames, uint64_t frame_stride, uint32_t v_size, uint32_t u_size);

/* encode_hex_mold_scaled (src/encode/write/mod.rs:190-217): a 1 at every
 * offset of gen_syn_offs(radius, calc_scale(frame, source)) around the
 * frame's middle; other bytes are left alone. A mold that would leave the
 * frame is refused. */
int bm_encode_hex_mold(bm_ctx ctx, int32_t radius, uint32_t src_v_size, uint32_t src_u_size, uint8_t* frame,
                       uint32_t v_size, uint32_t u_size);

/* encode_scalar (src/encode/write/mod.rs:28-172): each of n values (host,
 * n <= 4096, within [lo, hi], hi > 0) clears its frame and draws a hexagon
 * of radius (v + u) / 32 of bytes in 64..127 along the frame's border. */
int bm_encode_scalar(bm_ctx ctx, const float* vals, uint32_t n, float lo, float hi, uint64_t seed, uint8_t* frames,
                     uint64_t frame_stride, uint32_t v_size, uint32_t u_size);

/* ScalarGlyphWriter (src/encode/write/scalar_glyph_writer.rs:25-151), which
 * VectorEncoder and ScalarSequence write with: each of n values (host,
 * n <= 4096, within [lo, hi]) clears its frame and sets to 127 the hexagon of
 * radius (v + u) / 32 around the value's tile on a track along the frame's
 * margin (clockwise from the upper left). */
int bm_encode_scalar_glyph(bm_ctx ctx, const float* vals, uint32_t n, float lo, float hi, uint8_t* frames,
                           uint64_t frame_stride, uint32_t v_size, uint32_t u_size);

/* ScalarSdrWriter (src/encode/write/scalar_sdr_writer.rs:96-235): waypoint
 * SDRs every `way_span` across [lo, hi], each v*u/48 seeded axon indices
 * (held on the device); encode blends the two waypoints around each value. */
typedef struct bm_sdr_writer_s* bm_sdr_writer;
int bm_sdr_writer_create(bm_ctx ctx, float lo, float hi, float way_span, uint32_t v_size, uint32_t u_size,
                         uint64_t seed, bm_sdr_writer* out);
int bm_sdr_writer_destroy(bm_sdr_writer w);
int bm_sdr_writer_info(bm_sdr_writer w, uint32_t* way_count, uint32_t* active, uint32_t* len);
/* The waypoint table (way_count x active indices) into host memory. */
int bm_sdr_writer_waypoints(bm_sdr_writer w, uint32_t* dst, uint64_t n);
/* n values (host, n <= 2048) -> n frames (device). */
int bm_sdr_writer_encode(bm_sdr_writer w, const float* vals, uint32_t n, uint8_t* frames, uint64_t frame_stride);

#ifdef __cplusplus
}
#endif

#endif /* BISMIT_B200_H */
