/*
 * bm3d_b200.h -- C ABI of the B200-native BM3D / V-BM3D library (sm_100a).
 *
 * Drop-in boundary for the reference VapourSynth plugin "bm3d" (id com.vapoursynth.bm3d, v10.1).
 * The reference exposes seven functions through VapourSynthPluginInit2 (source/VSPlugin.cpp:424-518):
 * RGB2OPP, OPP2RGB, Basic, Final, VBasic, VFinal, VAggregate.  Each is created from a VSMap of
 * arguments (the *_Create callbacks, source/VSPlugin.cpp:64-417), produces frames on request (the
 * *_GetFrame callbacks) and is released by *_Free.  This header mirrors that life cycle with plain
 * C types:
 *
 *   bm3d_map_*         <-> VSMap argument passing (mapSetInt/Float/Data/Node,
 *                          mapGetIntSaturated/mapGetFloat/mapGetData/mapNumElements semantics)
 *   bm3d_create        <-> <Func>_Create + <Func>_Data::arguments_process (same argument names,
 *                          defaults, validation order and error text "bm3d.<Func>: <msg>")
 *   bm3d_frame_window  <-> the frame requests of <Func>_GetFrame(arInitial)
 *   bm3d_get_frames    <-> <Func>_GetFrame(arAllFramesReady) -> <Func>_Process::process(), for a
 *                          batch of consecutive output frames
 *   bm3d_free          <-> <Func>_Free
 *
 * Frames may live in host memory (the library stages them through the device) or in device
 * memory (no copies; frames stay on the GPU between stages).  All arithmetic runs on the GPU;
 * there is no CPU fallback: without a usable CUDA device every call fails with BM3D_ERR_CUDA.
 */
#ifndef BM3D_B200_H
#define BM3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define BM3D_API __declspec(dllexport)
#else
#define BM3D_API __attribute__((visibility("default")))
#endif

#define BM3D_B200_ABI_VERSION 1

/* Status codes.  Every failing call records a message readable with bm3d_get_error(). */
enum {
    BM3D_OK = 0,
    BM3D_ERR_ARG = 1,          /* invalid argument (the reference's mapSetError path) */
    BM3D_ERR_CUDA = 2,         /* CUDA runtime error or no device */
    BM3D_ERR_UNSUPPORTED = 3,  /* parameters beyond this build's limits */
    BM3D_ERR_STATE = 4         /* misuse of the API (null pointers, wrong frame count, ...) */
};

/* VapourSynth enumerations, same values (VSColorFamily, VSSampleType). */
enum { BM3D_GRAY = 1, BM3D_RGB = 2, BM3D_YUV = 3 };
enum { BM3D_INTEGER = 0, BM3D_FLOAT = 1 };
enum { BM3D_MEM_HOST = 0, BM3D_MEM_DEVICE = 1 };

/* Clip description (VSVideoInfo with its VSVideoFormat flattened). */
typedef struct bm3d_video_info {
    int color_family;      /* BM3D_GRAY / BM3D_RGB / BM3D_YUV */
    int sample_type;       /* BM3D_INTEGER / BM3D_FLOAT */
    int bits_per_sample;   /* 8..16 for integer, 32 for float */
    int subsampling_w;
    int subsampling_h;
    int width;
    int height;
    int num_frames;
} bm3d_video_info;

/* One frame: up to three planes plus the frame properties the reference reads and writes
 * (include/BM3D_Base.h:189-223, include/VBM3D_Base.h:252-312, include/VAggregate.h:147-231,
 * include/RGB2OPP.h:171-180, include/OPP2RGB.h:171-180).  A property value of -1 means "absent". */
typedef struct bm3d_frame {
    void *data[3];
    int64_t stride[3];          /* bytes between rows */
    int memory;                 /* BM3D_MEM_HOST or BM3D_MEM_DEVICE */
    int64_t prop_bm3d_opp;      /* "BM3D_OPP" */
    int64_t prop_range;         /* "_Range" */
    int64_t prop_matrix;        /* "_Matrix" */
    int64_t prop_v_radius;      /* "BM3D_V_radius" */
    int64_t prop_v_process[3];  /* "BM3D_V_process" (valid when prop_v_process_count == 3) */
    int prop_v_process_count;   /* number of elements, -1 if absent */
} bm3d_frame;

/* Argument map (VSMap analogue).  Keys are the reference argument names
 * (source/VSPlugin.cpp:430-517).  Arrays are built by repeated set calls. */
typedef struct bm3d_map bm3d_map;

BM3D_API bm3d_map *bm3d_map_create(void);
BM3D_API void bm3d_map_free(bm3d_map *map);
BM3D_API int bm3d_map_set_int(bm3d_map *map, const char *key, int64_t value);
BM3D_API int bm3d_map_set_float(bm3d_map *map, const char *key, double value);
BM3D_API int bm3d_map_set_data(bm3d_map *map, const char *key, const char *value);
BM3D_API int bm3d_map_set_clip(bm3d_map *map, const char *key, const bm3d_video_info *clip);

typedef struct bm3d_filter bm3d_filter;

/* Creates a filter.  name is one of "RGB2OPP", "OPP2RGB", "Basic", "Final", "VBasic", "VFinal",
 * "VAggregate" (VapourSynthPluginInit2, source/VSPlugin.cpp:430-517).  On invalid arguments
 * returns BM3D_ERR_ARG with the reference's message, e.g.
 * "bm3d.Basic: Invalid \"block_size\" assigned, must be an integer in [1, 64]"
 * (source/BM3D_Base.cpp:32-259, source/VBM3D_Base.cpp:104-379, source/VAggregate.cpp:32-86,
 * include/RGB2OPP.h:55-96, include/OPP2RGB.h:55-96). */
BM3D_API int bm3d_create(const char *name, const bm3d_map *args, bm3d_filter **out);

/* Output clip description (the VSVideoInfo passed to createVideoFilter). */
BM3D_API int bm3d_output_info(const bm3d_filter *filter, bm3d_video_info *out);

/* Input frames needed to produce output frames [n, n + count): clip frames
 * [*first, *first + *num) of the input (and of ref).  For VBasic / VFinal / VAggregate this is the
 * +-radius window clamped to the clip (VBM3D_Basic_GetFrame, source/VSPlugin.cpp:238-263). */
BM3D_API int bm3d_frame_window(const bm3d_filter *filter, int n, int count, int *first, int *num);

/* Produces output frames [n, n + count).  src[i] (and ref[i] when the filter has a ref clip) is
 * clip frame first + i of the window returned by bm3d_frame_window; dst[k] receives output frame
 * n + k.  Planes of dst must be allocated by the caller with the output format.  Output frame
 * properties are written into dst.  Blocks until the results are in dst. */
BM3D_API int bm3d_get_frames(bm3d_filter *filter, int n, int count, const bm3d_frame *const *src,
                             const bm3d_frame *const *ref, bm3d_frame *const *dst);

/* Same as bm3d_get_frames but returns after enqueuing the work on the filter's stream when all
 * frames are in device memory (call bm3d_synchronize before reading dst). */
BM3D_API int bm3d_get_frames_async(bm3d_filter *filter, int n, int count, const bm3d_frame *const *src,
                                   const bm3d_frame *const *ref, bm3d_frame *const *dst);

/* Selects the CUDA stream (a cudaStream_t) the filter enqueues on; NULL restores its own stream. */
BM3D_API int bm3d_set_stream(bm3d_filter *filter, void *cuda_stream);
BM3D_API int bm3d_synchronize(bm3d_filter *filter);

BM3D_API void bm3d_free(bm3d_filter *filter);

/* Last error message of the calling thread ("" if none). */
BM3D_API const char *bm3d_get_error(void);

/* Warnings the reference logs with vsapi->logMessage(mtWarning, ...) go to this callback
 * (default: stderr). */
typedef void (*bm3d_log_fn)(int level, const char *message, void *user);
BM3D_API void bm3d_set_log_callback(bm3d_log_fn fn, void *user);

/* ---- allocation-free Basic estimate of one plane ----------------------------------------------
 * No counterpart in the reference (the plugin allocates its buffers per frame).  For callers that
 * cannot let a library call cudaMalloc: hosts that give all of the GPU's memory to their own pool
 * allocator at start-up, where an outside allocation fails or breaks their accounting, and
 * real-time pipelines that forbid cudaMalloc / cudaFree because those calls synchronise the whole
 * device.  The filter objects above allocate workspaces on first use; this call allocates nothing.
 *
 * Computes bm3d.Basic(clip, profile=profile, sigma=sigma) for one 32-bit float GRAY plane, every
 * other argument at its default.  src and dst are device pointers with `stride` bytes between
 * rows (a multiple of 4, at least width * 4); profile NULL means "fast".  Work is queued on
 * `stream` (a cudaStream_t; NULL is the legacy default stream) and the call returns without
 * waiting for it.
 *
 * Its work buffers are one fixed 48 MiB device array inside the library, held by every GPU that
 * loads the library's device code until the process exits.  A plane that needs more (1920x1080
 * fits at every profile; a 3840x2160 plane does not) is rejected with BM3D_ERR_UNSUPPORTED and a
 * message that gives the size it needed.  The first call on a device sets that device up (finds the
 * array's device address and copies constant tables with synchronous copies): make that first call
 * before any stream capture on the device.  All calls share the one array, which keeps the last
 * call's contents; each call clears what must start at zero, but calls that overlap on the GPU
 * (different streams, or host threads that do not order their calls) race and corrupt each
 * other's results, so order them on one stream.  The set-up is not redone after a device reset:
 * do not call cudaDeviceReset on a device after the first call on it. */
BM3D_API int bm3d_basic_noalloc(const float *src, float *dst, int width, int height, int64_t stride,
                                const char *profile, double sigma, void *cuda_stream);

/* ---- inspection entry points (tests and tooling) ---------------------------------------------
 * Match lists of the last bm3d_get_frames call of a Basic/Final/VBasic/VFinal filter, for output
 * frame k of that batch, in reference-block scan order (row-major over the clamped scan of
 * source/BM3D_Base.cpp:421-443).  Per block: count, then up to group_size entries of
 * (z, y, x, key); z is the window frame index (0 for BM3D).  Returns the number of blocks, or -1. */
BM3D_API int bm3d_debug_matches(bm3d_filter *filter, int k, int *counts, int *zs, int *ys, int *xs,
                                float *keys, int capacity_blocks);
/* Stage timing with CUDA events on the filter's stream (off by default).  After a call with
 * profiling enabled, bm3d_debug_stage_times writes the durations in milliseconds of its stages:
 * [0] input conversion, [1] block matching, [2] predictive search (V-BM3D), [3] collaborative
 * filter + aggregation, [4] normalisation / stacking, [5] output conversion.  Returns the number
 * of stages written (0 when nothing was recorded). */
BM3D_API int bm3d_set_profiling(bm3d_filter *filter, int enable);
BM3D_API int bm3d_debug_stage_times(bm3d_filter *filter, double *ms, int capacity);
/* FP64 GPU oracle: frame k of the last bm3d_get_frames call of a Basic or Final filter recomputed
 * in double precision from the filter's own match lists -- 3-D DCTs, hard threshold or Wiener
 * shrinkage, aggregation and normalisation (source/BM3D_Basic.cpp:72-148,
 * source/BM3D_Final.cpp:50-127, source/BM3D_Base.cpp:348-351), thresholds and variances in double.
 * Writes the processed planes of the internal float domain (the filter's output before any
 * output-format conversion) as doubles to HOST memory, planes[p * plane_stride + y * width + x].
 * Returns 0, or -1 (V-BM3D filter, no such frame, or block/group size beyond its shared memory).
 * An inspection tool for the error of the FP32 and tf32 forms; it allocates device memory. */
BM3D_API int bm3d_debug_reference_fp64(bm3d_filter *filter, int k, double *planes, int64_t plane_stride);
/* Number of kernels this library has launched since it was loaded (all filters). */
BM3D_API int64_t bm3d_debug_launch_count(void);
/* Number of reference blocks that took the exact tie-resolution path in the last call. */
BM3D_API int64_t bm3d_debug_slow_blocks(bm3d_filter *filter);
/* Precision form ("tf32") block matching of the last call: reference blocks whose tensor-core
 * distance estimates could not settle the list (all distances then computed exactly), and CTAs
 * whose tensor-core wait timed out (their blocks also computed exactly).  No reference
 * counterpart.  Returns 0, or -1 for a null filter. */
BM3D_API int bm3d_debug_bm_tc_counts(bm3d_filter *filter, int64_t *fallbacks, int64_t *timeouts);
/* Precision form ("tf32"), hard threshold (Basic / VBasic), last call: coefficients whose
 * tensor-core value lay within the recheck band of their threshold and were recomputed in fp32,
 * and the keep / zero decisions that recomputation changed.  No reference counterpart (the
 * reference's threshold rule is source/BM3D_Basic.cpp:98-134).  Returns 0, or -1. */
BM3D_API int bm3d_debug_threshold_rechecks(bm3d_filter *filter, int64_t *rechecked, int64_t *changed);
/* Sets that band (a fraction of each coefficient's threshold; 0 disables the recheck). */
BM3D_API int bm3d_debug_set_recheck_band(bm3d_filter *filter, float band);
/* Retained-coefficient count of every group of output frame k of the last call of a Basic
 * filter (the count the reference turns into the group weight, source/BM3D_Basic.cpp:125-146),
 * as counts[plane * nblocks + block] in reference-block scan order, -1 for planes not processed.
 * Returns nblocks, or -1 (not a Basic filter, no such frame, capacity < 3 * nblocks). */
BM3D_API int bm3d_debug_retained_counts(bm3d_filter *filter, int k, int *counts, int capacity);
/* In-place 3-D transform of ngroups groups of n blocks of B x B floats in HOST memory (layout
 * [group][z][y][x]) using the device code of the collaborative filter; fast = 1 selects the
 * register path of the 8x8 / n in {8,16,32} kernels.  inverse = 0 forward (REDFT10 definition),
 * 1 inverse (REDFT01). */
BM3D_API int bm3d_debug_dct3d(float *groups, int ngroups, int n, int block_size, int inverse, int fast);

/* ---- Learned block-matching proposal (precision = "learned"); no reference counterpart --------
 * Network: 3x3 conv 1 -> 16 channels, ReLU, 3x3 conv 16 -> 16, bf16 activations; descriptor of
 * a block position = the 16 features averaged over its 8x8 block.  Weight vector (2480 floats):
 * w1[16][9], b1[16], w2[16][16][9], b2[16].  Planes are float GRAY, pitch = width.  All return 0
 * on success (match: the number of reference blocks) or an error code (bm3d_get_error). */
/* Copies the built-in (trained) weights; returns their count. */
BM3D_API int bm3d_proposal_default_weights(float *out, int capacity);
/* Descriptors [height - 7][width - 7][16] (bf16 values as float) of one plane. */
BM3D_API int bm3d_proposal_descriptors(const float *frame, int width, int height, const float *weights, float *desc_out);
/* Mean logistic ranking loss softplus(s_ap - s_an) over triplets (ay, ax, py, px, ny, nx) of block
 * positions, s = squared descriptor distance, and its gradient with respect to the weights. */
BM3D_API int bm3d_proposal_gradients(const float *frame, int width, int height, const float *weights, const int *triplets,
                                     int ntriplets, float *loss, float *grad);
/* Trains on nframes planes [n][height][width] for iters Adam steps of batch triplets; weights in
 * (initial) and out (trained); losses[iters] receives the mean loss of every step. */
BM3D_API int bm3d_proposal_train(const float *frames, int nframes, int width, int height, int iters, int batch, float lr,
                                 uint64_t seed, float *weights, float *losses);
/* Match lists of one plane (block step, group size <= 32, range, candidate step 1, SSD threshold):
 * exhaustive when weights is NULL, else the nprop (<= 128) best candidates by descriptor distance
 * re-ranked with the exact SSD.  counts[n], ys / xs [n][group_size]; capacity = room for n. */
BM3D_API int bm3d_proposal_match(const float *frame, int width, int height, const float *weights, int block_step,
                                 int group_size, int bm_range, float th_sse, int nprop, int *counts, int *ys, int *xs,
                                 int capacity);
/* Proposal sets of that matching (weights required): per reference block the nprop candidate
 * indices (raster order of its search window; the trailing default (0, 0) candidate of the
 * reference's search list is index (window size)) whose exact distances are taken, unused slots
 * 0xffffffff; *overflow_blocks = blocks whose cut needed the exact bisection.  Returns the number
 * of reference blocks. */
BM3D_API int bm3d_debug_proposal_sets(const float *frame, int width, int height, const float *weights, int block_step,
                                      int bm_range, int nprop, uint32_t *sets, int64_t *overflow_blocks, int capacity);

#ifdef __cplusplus
}
#endif

#endif /* BM3D_B200_H */
