/* bmfr_batch.h — many BMFR streams denoised together on one GPU.
 *
 * The reference denoises one stream on one in-order queue
 * (opencl/bmfr.cpp:191, 417-485); this layer has no counterpart there.  A
 * batch holds the temporal history of many streams of uneven resolution in
 * HBM and denoises one frame of any subset of them per step: the steps's
 * 32x32 blocks of all those streams form one queue that a single persistent
 * launch walks, and the whole step is one CUDA graph.  Each stream's result
 * is exactly what a plan with the same parameters and the fused pipeline
 * produces for it alone.
 *
 * A server on top admits render streams against a memory budget, queues
 * their frame requests as they arrive and runs steps continuously, so that
 * requests arriving while a step is on the GPU join the next one.
 *
 * Conventions as in bmfr_b200.h: status codes, asynchronous calls on a CUDA
 * stream, device pointers unless stated otherwise.
 */
#ifndef BMFR_BATCH_H
#define BMFR_BATCH_H

#include <stddef.h>
#include <stdint.h>

#include "bmfr_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define BMFR_BATCH_MAX_STREAMS 128

typedef struct bmfr_batch bmfr_batch;

/* Launch parameters of a step, chosen by bmfr_batch_autotune. */
typedef struct bmfr_batch_tuning {
    int block_ctas_per_sm;  /* persistent CTAs of the block kernel per SM (0: as many as fit) */
    int taa_tile_w;         /* TAA CTA shape: 32x8, 32x4, 64x4 or 16x16 */
    int taa_tile_h;
    int staging_depth;      /* 0: blocks from an atomic queue; k > 0: static order with the
                               inputs of each CTA's next k blocks prefetched into L2 */
} bmfr_batch_tuning;

/* memory_budget_bytes: device bytes the batch's streams may hold (0: no limit).
 * params: shared by every stream; the batch always runs the fused pipeline. */
int bmfr_batch_create(const bmfr_params* params, size_t memory_budget_bytes, bmfr_batch** batch);
int bmfr_batch_destroy(bmfr_batch* batch);

/* Device bytes a stream of this size holds (histories, per-frame buffers and,
 * with own_inputs, the input slots). */
int bmfr_batch_stream_bytes(const bmfr_params* params, int width, int height, int own_inputs,
                            size_t* bytes);

/* Adds a stream (frame counter 0); BMFR_E_BUDGET if it does not fit in the
 * budget, BMFR_E_TOO_LARGE past BMFR_BATCH_MAX_STREAMS.  own_inputs: the batch
 * also allocates input slots for it (bmfr_batch_stream_inputs); otherwise
 * every step must name the caller's input buffers. */
int bmfr_batch_add_stream(bmfr_batch* batch, int width, int height, int own_inputs, int* slot);
int bmfr_batch_remove_stream(bmfr_batch* batch, int slot);
/* Frame counter back to 0: the stream's next frame starts a new sequence. */
int bmfr_batch_reset_stream(bmfr_batch* batch, int slot);
int bmfr_batch_stream_frame(const bmfr_batch* batch, int slot);
size_t bmfr_batch_bytes_in_use(const bmfr_batch* batch);

/* Device slots for the stream's next frame (own_inputs streams only). */
int bmfr_batch_stream_inputs(bmfr_batch* batch, int slot, bmfr_frame_inputs* inputs);

/* One step: frame number bmfr_batch_stream_frame(slot) of each of the n
 * listed streams.  io: n entries of caller buffers, or NULL (every listed
 * stream then uses its own input slots); an entry whose albedo is NULL also
 * uses the stream's slots.  matrices: n * 16 floats (each stream's
 * camera_matrices[max(f-1,0)]); offsets: n * 2 floats; both host memory.
 * Steps of one batch run in call order (each waits for the previous). */
int bmfr_batch_step(bmfr_batch* batch, int n, const int* slots, const bmfr_frame_io* io,
                    const float* matrices, const float* offsets, void* stream);

/* Float output of the stream's last denoised frame (device, W*H*3). */
int bmfr_batch_stream_result(const bmfr_batch* batch, int slot, const float** result);

int bmfr_batch_get_tuning(const bmfr_batch* batch, bmfr_batch_tuning* tuning);
int bmfr_batch_set_tuning(bmfr_batch* batch, const bmfr_batch_tuning* tuning);
/* Times candidate tunings on `steps` steps of the given work (which advances
 * the listed streams' histories; reset them afterwards if that matters),
 * keeps the fastest and returns it with its mean step time. */
int bmfr_batch_autotune(bmfr_batch* batch, int n, const int* slots, const bmfr_frame_io* io,
                        const float* matrices, const float* offsets, int steps, void* stream,
                        bmfr_batch_tuning* chosen, float* best_ms);

#ifdef __cplusplus
}
#endif
#endif /* BMFR_BATCH_H */
