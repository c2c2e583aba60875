/* bmfr_b200.h — C ABI of the B200 (sm_100a) BMFR denoising pipeline.
 *
 * The five per-frame stages of Blockwise Multi-Order Feature Regression keep
 * the argument order, element types and buffer sizes of the reference's
 * OpenCL kernels (opencl/bmfr.cl:290-308, 490-501, 703-710, 761-770,
 * 860-865), bound by the reference host at opencl/bmfr.cpp:349-384 and
 * 429-476.  The reference's compile-time -D options (opencl/bmfr.cpp:205-232)
 * become the runtime struct bmfr_params plus the fixed constants below.
 *
 * Conventions for every entry point:
 *  - pointers named in the kernel argument lists are DEVICE memory owned by
 *    the caller (the reference host allocates every buffer,
 *    opencl/bmfr.cpp:315-347); no kernel entry point allocates;
 *  - the call is asynchronous on the given CUDA stream (a cudaStream_t; 0 is
 *    the legacy default stream) and is thread-safe across distinct streams;
 *  - the return value is BMFR_OK (0) or a negative BMFR_E_* status.  The
 *    reference reported failures as cl::Error exceptions caught in main
 *    (opencl/bmfr.cpp:558-577); bmfr_last_error() gives the message of the
 *    last failure on the calling thread.
 *
 * Float buffers of three channels use the reference's interleaved layout
 * (pixel i at [3i, 3i+2]), row-major with the IMAGE width as stride, exactly
 * as load_float3/store_float3 (opencl/bmfr.cl:224-241) index them.
 */
#ifndef BMFR_B200_H
#define BMFR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Fixed layout constants (opencl/bmfr.cpp:56-118, 193-232). */
#define BMFR_BLOCK_EDGE_LENGTH 32   /* BLOCK_EDGE_LENGTH, bmfr.cpp:104        */
#define BMFR_BLOCK_PIXELS 1024      /* BLOCK_PIXELS, bmfr.cpp:105             */
#define BMFR_LOCAL_SIZE 256         /* fitter work-group size, bmfr.cpp:116   */
#define BMFR_FEATURES_NOT_SCALED 4  /* 1, n.x, n.y, n.z  (bmfr.cpp:65-69)     */
#define BMFR_FEATURES_SCALED 6      /* p.xyz, p.xyz^2    (bmfr.cpp:71-77)     */
#define BMFR_FEATURE_COUNT 10       /* BUFFER_COUNT - 3                       */
#define BMFR_BUFFER_COUNT 13        /* 10 features + 3 colour channels        */
#define BMFR_R_EDGE 11              /* BUFFER_COUNT - 2, bmfr.cpp:221         */
#define BMFR_BLOCK_OFFSETS_COUNT 16 /* bmfr.cl:267                            */

/* Status codes. */
#define BMFR_OK 0
#define BMFR_E_INVALID -1       /* bad argument (null pointer, size, frame)  */
#define BMFR_E_CUDA -2          /* a CUDA runtime call failed                */
#define BMFR_E_UNSUPPORTED -3   /* parameter value this build does not serve */
#define BMFR_E_NOMEM -4         /* device allocation failed                  */
#define BMFR_E_BUDGET -5        /* server admission over the memory budget   */
#define BMFR_E_NOT_FOUND -6     /* unknown stream / request id               */
#define BMFR_E_AGAIN -7         /* nothing ready yet (poll again)            */
#define BMFR_E_TIMEOUT -8       /* a bounded wait ran out                    */
#define BMFR_E_STATE -9         /* call not valid in the object's state      */
#define BMFR_E_TOO_LARGE -10    /* size beyond a fixed maximum               */

/* Pipeline variants of bmfr_denoise_frame / bmfr_batch_step. */
#define BMFR_PIPELINE_STAGED 0  /* the five stage kernels, reference order   */
#define BMFR_PIPELINE_FUSED 1   /* accumulate+fit in one kernel per 32x32
                                   block (tmp_data stays on chip), then
                                   weighted sum+filtered accumulation, then
                                   TAA                                       */

/* Runtime form of the reference's compile-time options.  Defaults
 * (bmfr_params_default) are the reference's values.  */
typedef struct bmfr_params {
    double noise_amount;           /* NOISE_AMOUNT 1e-2 (bmfr.cpp:58); a double
                                   literal in the reference, so the noise
                                   term is formed in double precision       */
    float blend_alpha;             /* BLEND_ALPHA 0.2 (bmfr.cpp:60)            */
    float second_blend_alpha;      /* SECOND_BLEND_ALPHA 0.1 (bmfr.cpp:61)     */
    float taa_blend_alpha;         /* TAA_BLEND_ALPHA 0.2 (bmfr.cpp:62)        */
    float position_limit_squared;  /* from the dataset's camera_matrices.h,   */
    float normal_limit_squared;    /*   bmfr.cpp:226-227                       */
    int use_half_precision_in_tmp_data; /* 1 (bmfr.cpp:88): tmp_data is
                                   binary16; 0: float32                      */
    int compressed_r;              /* 1 (bmfr.cpp:82); accepted, R is internal */
    int cache_tmp_data;            /* 1 (bmfr.cpp:84); 0 is not served         */
    int fp32_qr;                   /* the fit's arithmetic (binary16 tmp_data):
                                   0 the reference's Householder sequence,
                                   rounding every in-place tmp update to
                                   binary16 (bmfr.cl:540, 651); precision
                                   form, the block in FP32 registers:
                                   1 CholeskyQR2 (BMFR_QR_CHOLESKY2),
                                   2 the Householder sequence (BMFR_QR_HOUSEHOLDER) */
    int half_history;              /* precision form, plan pipeline only: the
                                   colour histories are stored as binary16   */
    int pipeline;                  /* BMFR_PIPELINE_* for bmfr_denoise_frame   */
} bmfr_params;

#define BMFR_QR_REFERENCE 0
#define BMFR_QR_CHOLESKY2 1
#define BMFR_QR_HOUSEHOLDER 2

/* Sizes derived by bmfr_plan_create (bmfr.cpp:104-118, 315-347). */
typedef struct bmfr_sizes {
    int image_width, image_height;       /* IMAGE_WIDTH/HEIGHT                 */
    int workset_width, workset_height;   /* rounded up to 32                   */
    int margin_width, margin_height;     /* WORKSET_WITH_MARGINS_* (+32)       */
    int blocks_x, blocks_y, blocks;      /* fitter work-groups                 */
    size_t tmp_data_bytes;               /* margin px * 13 * sizeof(tmp type)  */
    size_t weights_bytes;                /* blocks * 10 * 3 floats             */
    size_t mins_maxs_bytes;              /* blocks * 6 * 2 floats              */
    size_t pixel3_bytes;                 /* W * H * 3 floats                   */
} bmfr_sizes;

typedef struct bmfr_plan bmfr_plan;

int bmfr_params_default(bmfr_params* params);
/* Derives workset, margin and block counts; the plan also owns the history
 * buffers of the frame pipeline (the reference's six Double_buffers and eight
 * single buffers, bmfr.cpp:122-135, 315-347), allocated on the current device.
 * Width and height must exceed 32 (mirror(), bmfr.cl:207-222, is valid for at
 * most one image size out of bounds). */
int bmfr_plan_create(const bmfr_params* params, int width, int height, bmfr_plan** plan);
int bmfr_plan_destroy(bmfr_plan* plan);
int bmfr_plan_sizes(const bmfr_plan* plan, bmfr_sizes* sizes);
int bmfr_plan_params(const bmfr_plan* plan, bmfr_params* params);

/* The reference's constant BLOCK_OFFSETS table (bmfr.cl:267-285), as 16 int2. */
int bmfr_block_offsets(int out_xy[32]);

/* ---- the five stages (drop-in for the reference's kernels) -------------- */

/* accumulate_noisy_data (bmfr.cl:290-485).  current_noisy is read and then
 * overwritten in place with the blended colour for in-image pixels, as in the
 * reference.  The margin threads that mirror an in-image pixel use the same
 * blended colour as that pixel's own thread (the reference reads the buffer
 * while other threads write it, bmfr.cl:322 and 481; here the result is
 * defined).  tmp_data is binary16 or float32 per
 * params.use_half_precision_in_tmp_data, laid out [block][13][1024].
 * prev_frame_camera_matrix: 16 floats as the reference's float16 argument
 * (camera_matrices[max(f-1,0)], bmfr.cpp:440-442).  pixel_offset: 2 floats
 * (pixel_offsets[f], bmfr.cpp:443-444).  Both are host pointers.  */
int bmfr_accumulate_noisy_data(const bmfr_plan* plan,
                               float* out_prev_frame_pixel,   /* float2[W*H] */
                               uint8_t* accept_bools,         /* [W*H]       */
                               const float* current_normals,
                               const float* previous_normals,
                               const float* current_positions,
                               const float* previous_positions,
                               float* current_noisy,          /* in/out      */
                               const float* previous_noisy,
                               const uint8_t* previous_spp,
                               uint8_t* current_spp,
                               void* tmp_data,
                               const float* prev_frame_camera_matrix,
                               const float* pixel_offset,
                               int frame_number,
                               void* stream);

/* fitter (bmfr.cl:490-700): per 32x32 block, min/max scaling of the six
 * position features, Householder QR of the 1024x13 block and back
 * substitution.  Writes weights[block][10][3] and mins_maxs[block][6][2].
 * tmp_data is read only; the reference leaves QR intermediates in it that no
 * later stage reads (bmfr.cl:540, 651). */
int bmfr_fitter(const bmfr_plan* plan, float* weights, float* mins_maxs,
                const void* tmp_data, int frame_number, void* stream);

/* The fitter in double precision, the reference arithmetic of the
 * precision form (params.fp32_qr): same steps, reduction trees and noise as
 * bmfr_fitter, every value in double and no intermediate rounding.  weights:
 * blocks * 10 * 3 doubles.  The only FP64 code on the device. */
int bmfr_fitter_fp64(const bmfr_plan* plan, double* weights, float* mins_maxs,
                     const void* tmp_data, int frame_number, void* stream);

/* bmfr_fitter without any device allocation; no counterpart in the
 * reference.  For callers that cannot call cudaMalloc: renderers whose engine
 * owns all device memory under a fixed budget, and per-frame code that cannot
 * afford cudaMalloc's implicit device synchronisation.  It needs no plan
 * (creating one allocates the history buffers): the sizes come from
 * width/height and the options from params.  The fitter's scratch — the
 * frame's noise table and a status word, 37,120 bytes — lives in a static
 * device array of the library that every GPU loading the library holds until
 * the process exits; its size does not grow with the image, so every size a
 * plan accepts is served and larger sizes are rejected like plan creation
 * rejects them.  The first call on a device looks up that array's device
 * address (cudaGetSymbolAddress) with the device current; make that first
 * call before any stream capture.  All calls share the array and each call
 * rewrites it, so calls whose kernels overlap on the GPU (different streams,
 * or one stream and another without ordering) race: order them.  The
 * weights and min/max values are bit for bit those of bmfr_fitter (the same
 * arithmetic).  A bounded wait that runs out is recorded in the array's
 * status word, which no call clears; bmfr_fitter_noalloc_check reads it. */
int bmfr_fitter_noalloc(const bmfr_params* params, int width, int height,
                        float* weights, float* mins_maxs, const void* tmp_data,
                        int frame_number, void* stream);
/* Waits for `stream` and reports whether a bmfr_fitter_noalloc kernel on the
 * current device gave up a bounded wait since the last check
 * (BMFR_E_TIMEOUT; the status word is then cleared).  Allocates nothing. */
int bmfr_fitter_noalloc_check(void* stream);
/* Diagnostics of that failure path, as bmfr_plan_probe_bounded_wait for a
 * plan: one CTA whose bounded wait (limit_us, 1..1,000,000) on a barrier
 * that nothing completes runs out and records the timeout in the static
 * array's status word; no fault, trap or endless wait is involved. */
int bmfr_fitter_noalloc_probe_bounded_wait(unsigned int limit_us, void* stream);

/* weighted_sum (bmfr.cl:703-758). current_noisy is unused, as in the
 * reference (debug only, bmfr.cl:709), and may be NULL. */
int bmfr_weighted_sum(const bmfr_plan* plan, const float* weights,
                      const float* mins_maxs, float* output,
                      const float* current_normals,
                      const float* current_positions,
                      const float* current_noisy, int frame_number,
                      void* stream);

/* accumulate_filtered_data (bmfr.cl:761-857). */
int bmfr_accumulate_filtered_data(const bmfr_plan* plan,
                                  const float* filtered_frame,
                                  const float* in_prev_frame_pixel,
                                  const uint8_t* accept_bools,
                                  const float* albedo,
                                  float* tone_mapped_frame,
                                  const uint8_t* current_spp,
                                  const float* accumulated_prev_frame,
                                  float* accumulated_frame,
                                  int frame_number, void* stream);

/* taa (bmfr.cl:860-974). */
int bmfr_taa(const bmfr_plan* plan, const float* in_prev_frame_pixel,
             const float* new_frame, float* result_frame,
             const float* prev_frame, int frame_number, void* stream);

/* ---- plan-managed frame pipeline (the reference's frame loop,
 *      bmfr.cpp:417-485) ------------------------------------------------- */

/* Device pointers of the slots the caller fills for the next frame
 * (the reference's enqueueWriteBuffer targets, bmfr.cpp:420-427). */
typedef struct bmfr_frame_inputs {
    float* albedo;
    float* normals;
    float* positions;
    float* noisy;
} bmfr_frame_inputs;

int bmfr_plan_frame_inputs(bmfr_plan* plan, bmfr_frame_inputs* inputs);
/* Host-to-device copies of one frame's four buffers into those slots.
 * Uploads, bmfr_denoise_frame and bmfr_plan_download_result may be called on
 * three different streams: the plan keeps three input sets and two result
 * buffers and orders them with events, so that the upload of frame f+1 and
 * the download of frame f-1 overlap the denoising of frame f. */
int bmfr_plan_upload_frame(bmfr_plan* plan, const float* albedo,
                           const float* normals, const float* positions,
                           const float* noisy, void* stream);
/* Runs the five stages for frame plan->frame (params.pipeline selects the
 * staged or fused form), then swaps the double buffers (bmfr.cpp:482-484) and
 * advances the frame counter. */
int bmfr_denoise_frame(bmfr_plan* plan, const float* prev_frame_camera_matrix,
                       const float* pixel_offset, void* stream);
/* Caller-owned device buffers of one frame, for renderers that keep their own
 * G-buffers: the current frame's four inputs, the previous frame's normals and
 * positions (the reference's Double_buffer::previous(), bmfr.cpp:431-434),
 * and an optional extra copy of the output (NULL: only the plan's history
 * receives it).  Every pointer except result is read only. */
typedef struct bmfr_frame_io {
    const float* albedo;
    const float* normals;
    const float* positions;
    const float* noisy;
    const float* previous_normals;    /* may be NULL at frame 0 */
    const float* previous_positions;  /* may be NULL at frame 0 */
    float* result;                    /* optional, W*H*3 floats */
} bmfr_frame_io;

/* bmfr_denoise_frame on caller-owned input buffers instead of the plan's
 * slots; the histories stay in the plan. */
int bmfr_denoise_frame_io(bmfr_plan* plan, const bmfr_frame_io* io,
                          const float* prev_frame_camera_matrix,
                          const float* pixel_offset, void* stream);

/* The reference's frame loop (bmfr.cpp:417-485) over `count` consecutive
 * frames in one call: the same work and outputs, bit for bit, as count calls
 * of bmfr_denoise_frame_io with io[i], the 16 floats at
 * prev_frame_camera_matrices + 16*i and the 2 at pixel_offsets + 2*i.  The
 * call is ordered after the work already on `stream`, and work queued on
 * `stream` after it sees every frame's output (io[i].result where given; the
 * last frame's through bmfr_plan_result).  With the staged pipeline the
 * accumulation of frame i+1 runs while frame i's fitter, weighted sum and
 * TAA run, on two streams of the plan's own (the accumulation at the
 * device's lowest stream priority, the rest at its highest) forked from and
 * joined back into `stream`: the accumulation only needs frame i's
 * accumulated history, and the plan alternates two sets of the per-frame
 * buffers it writes (tmp_data, reprojected positions, accept mask, fitter
 * noise table).  The first such call allocates that second set (about 37 B
 * per pixel with binary16 tmp_data).  The buffers io[] points to must not be written while the
 * call's work runs.  The fused pipeline, and any call while stage profiling
 * is on, runs the frames one after another on `stream`.  Every frame's
 * arguments are checked before the first is queued; a CUDA error part way
 * through returns its status, and what was already queued on the plan's two
 * streams is still joined back into `stream`. */
int bmfr_denoise_frames(bmfr_plan* plan, int count, const bmfr_frame_io* io,
                        const float* prev_frame_camera_matrices,
                        const float* pixel_offsets, void* stream);

/* Device pointer of the last finished frame's TAA output (W*H*3 floats). */
int bmfr_plan_result(const bmfr_plan* plan, const float** result);
/* Device-to-host copy of the last finished frame's output; ordered after
 * that frame on any stream, and before the frame that reuses its buffer. */
int bmfr_plan_download_result(bmfr_plan* plan, float* host_rgb, void* stream);
int bmfr_plan_frame_number(const bmfr_plan* plan);
int bmfr_plan_reset(bmfr_plan* plan);   /* frame counter back to 0 */

/* Intermediate buffers of the last frame, for inspection and tests.  Which
 * pointers exist depends on the pipeline: the fused pipeline keeps no
 * tmp_data (NULL); both pipelines run weighted_sum and
 * accumulate_filtered_data as one kernel, whose filtered frame is written
 * (non-NULL here) only while bmfr_plan_keep_intermediates is on. */
typedef struct bmfr_plan_buffers {
    const void* tmp_data;
    const float* weights, *mins_maxs;
    const float* filtered, *prev_frame_pixel, *tone_mapped;
    const uint8_t* accept, *spp;
    const void* accumulated_noisy, *accumulated_filtered; /* f32 or f16 x3 */
    const float* result;
} bmfr_plan_buffers;
int bmfr_plan_buffers_get(const bmfr_plan* plan, bmfr_plan_buffers* buffers);
/* Enable (1) or disable (0, the default) writing the filtered frame of
 * every frame, which the reference keeps in a global buffer (bmfr.cpp:331)
 * and the plan otherwise keeps on chip between weighted_sum and
 * accumulate_filtered_data.  Outputs are the same either way. */
int bmfr_plan_keep_intermediates(bmfr_plan* plan, int enable);

/* Per-stage timing of the plan pipeline, in place of the reference's
 * per-kernel OpenCL event profiling (bmfr.cpp:386-412, 488-517).  While
 * enabled, every denoise call records CUDA events between its stages.
 * bmfr_plan_stage_times waits for the last frame and returns milliseconds of
 * the staged pipeline's [accumulate_noisy_data (with the frame's fitter
 * noise table), fitter, weighted_sum + accumulate_filtered_data (one kernel
 * in the plan pipeline), 0, taa].  The fused pipeline reports [noise table,
 * block kernel (accumulate and fitter), weighted_sum +
 * accumulate_filtered_data, 0, taa].  The five drop-in stage entry points
 * time separately with events around each call. */
#define BMFR_STAGE_COUNT 5
int bmfr_plan_enable_profiling(bmfr_plan* plan, int enable);
int bmfr_plan_stage_times(const bmfr_plan* plan, float ms[BMFR_STAGE_COUNT]);

/* Waits for `stream` and reports whether a kernel of this plan gave up a
 * bounded wait (BMFR_E_TIMEOUT; the device status is then cleared).  The
 * fitter waits on its bulk copies with a time limit instead of spinning
 * without end. */
int bmfr_plan_check_device(const bmfr_plan* plan, void* stream);

/* Diagnostics of the failure path above: enqueues on `stream` one CTA that
 * waits, with the fitter's bounded wait limited to `limit_us`
 * (1..1,000,000), on a barrier that nothing completes.  The wait runs out,
 * the timeout lands in the plan's device status, and the next
 * bmfr_plan_check_device returns BMFR_E_TIMEOUT; the plan and the CUDA
 * context stay usable.  No fault, trap or endless wait is involved. */
int bmfr_plan_probe_bounded_wait(bmfr_plan* plan, unsigned int limit_us, void* stream);

/* Error text of the last failing call on this thread ("" if none). */
const char* bmfr_last_error(void);
const char* bmfr_status_string(int status);

#ifdef __cplusplus
}
#endif
#endif /* BMFR_B200_H */
