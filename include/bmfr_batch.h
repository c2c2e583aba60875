/* bmfr_batch.h — many BMFR streams denoised together on one GPU.
 *
 * The reference denoises one stream on one in-order queue
 * (opencl/bmfr.cpp:191, 417-485); this layer has no counterpart there.  A
 * batch holds the temporal history of many streams of uneven resolution in
 * HBM and denoises one frame of any subset of them per step.  With
 * params.pipeline = BMFR_PIPELINE_FUSED the step is one CUDA graph: the
 * step's 32x32 blocks of all those streams form one queue that a single
 * persistent launch of the fused block kernel walks, and TAA follows in one
 * more launch.  With BMFR_PIPELINE_STAGED each listed stream runs a plan's
 * kernels (noise table, accumulation, fitter, weighted sum + filtered
 * accumulation, TAA) on its own buffers, the streams spread over eight worker
 * CUDA streams forked from and joined into the caller's stream, so that the
 * kernels of different streams overlap.  Each stream's result is exactly
 * what a plan with the same parameters (pipeline included) produces for it
 * alone.
 *
 * A server on top admits render streams against a memory budget, queues
 * their frame requests as they arrive and runs steps continuously, so that
 * requests arriving while a step is on the GPU join the next one.
 *
 * Conventions as in bmfr_b200.h: status codes, asynchronous calls on a CUDA
 * stream, device pointers unless stated otherwise.  Threads: steps, tuning
 * and autotuning of one batch are called from one thread at a time; streams
 * may be added, removed and reset from other threads meanwhile (stream
 * memory comes from a device pool in stream order, so adding or removing a
 * stream never synchronises the device).
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
    int block_ctas_per_sm;  /* fused step: persistent CTAs of the block kernel per SM
                               (0: as many as fit) */
    int taa_tile_w;         /* fused step's TAA CTA tile: 30 columns x 8, 16, 32 or 64 rows */
    int taa_tile_h;
    int staging_depth;      /* fused step: 0 takes blocks from an atomic queue; k > 0 a static
                               order with the inputs of each CTA's next k blocks prefetched
                               into L2.  The staged step launches a plan's kernels, whose
                               shapes are fixed: it has nothing to tune. */
    int pixel_pass;         /* fused step: 0 runs weighted sum + filtered accumulation in the
                               block kernel after each block's fit; 1 ends the block kernel at
                               the fit and runs them as a launch over every stream's 32x8
                               pixel tiles.  TAA follows either way. */
} bmfr_batch_tuning;

/* memory_budget_bytes: device bytes the batch's streams may hold (0: no limit).
 * params: shared by every stream (params.pipeline selects the step's form). */
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
/* Grows the batch's device memory pool to hold at least `bytes` (blocking),
 * so that streams added later take their memory from it without the pool
 * having to grow while steps run. */
int bmfr_batch_reserve(bmfr_batch* batch, size_t bytes);

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

/* Per-stream history snapshot, for moving a stream to another batch or GPU
 * between frames (no counterpart in the reference).  A snapshot holds the
 * stream's size and frame counter and the histories its next frame reads
 * (accumulated noisy and filtered colour, TAA result, spp; with input slots
 * the previous normals and positions).  bmfr_batch_snapshot copies it to
 * `dst` (host or device memory, bmfr_batch_snapshot_bytes long) after the
 * stream's last step and returns when the copy is done.  bmfr_batch_restore
 * adds a stream from a snapshot taken with the same history format
 * (half_history, tmp type) and returns its slot; its next frame continues
 * the sequence exactly as the original stream's would. */
int bmfr_batch_snapshot_bytes(const bmfr_batch* batch, int slot, size_t* bytes);
int bmfr_batch_snapshot(bmfr_batch* batch, int slot, void* dst, void* stream);
int bmfr_batch_restore(bmfr_batch* batch, const void* src, void* stream, int* slot);

/* Float output of the stream's last denoised frame (device, W*H*3). */
int bmfr_batch_stream_result(const bmfr_batch* batch, int slot, const float** result);

int bmfr_batch_get_tuning(const bmfr_batch* batch, bmfr_batch_tuning* tuning);
int bmfr_batch_set_tuning(bmfr_batch* batch, const bmfr_batch_tuning* tuning);
/* Times candidate tunings on `steps` steps of the given work (which advances
 * the listed streams' histories; reset them afterwards if that matters),
 * keeps the fastest and returns it with its mean step time (staged step:
 * only its time; the tuning stays as it is). */
int bmfr_batch_autotune(bmfr_batch* batch, int n, const int* slots, const bmfr_frame_io* io,
                        const float* matrices, const float* offsets, int steps, void* stream,
                        bmfr_batch_tuning* chosen, float* best_ms);

/* ---- server: continuous batching of frame requests ---------------------- */

typedef struct bmfr_server bmfr_server;

typedef struct bmfr_server_config {
    size_t memory_budget_bytes;  /* device bytes all streams may hold (0: no limit) */
    int max_streams_per_step;    /* at most this many frames per step (0: every stream that is ready) */
    int own_inputs;              /* streams get input slots (bmfr_server_stream_inputs) */
    int max_steps_in_flight;     /* steps launched and not finished before the next one is formed
                                    (0: 2, one running and one queued behind it) */
    size_t reserve_bytes;        /* stream memory to reserve at creation (bmfr_batch_reserve) */
} bmfr_server_config;

typedef struct bmfr_server_stats {
    uint64_t requests_submitted, requests_completed;
    uint64_t steps, frames;
    uint64_t streams_admitted, streams_rejected;
    double p50_latency_ms, p99_latency_ms, max_latency_ms, mean_latency_ms;
    double mean_frames_per_step;
    double busy_seconds;          /* wall time with at least one step in flight */
    double elapsed_seconds;       /* since the server started or the stats were reset */
} bmfr_server_stats;

/* Starts the server's scheduling thread on the current device.  Requests
 * that arrive while steps are on the GPU are queued and join the next step,
 * which is formed once fewer than max_steps_in_flight steps are outstanding;
 * each step takes the oldest pending frame of every ready stream.  Streams
 * join and leave without synchronising the device (their memory comes from
 * a stream-ordered pool). */
int bmfr_server_create(const bmfr_params* params, const bmfr_server_config* config, bmfr_server** server);
int bmfr_server_destroy(bmfr_server* server);   /* finishes queued work first */

/* Admits a render stream if its histories fit in the memory budget
 * (BMFR_E_BUDGET otherwise; retry once streams close). */
int bmfr_server_open_stream(bmfr_server* server, int width, int height, int* stream_id);
/* Waits for the stream's queued frames, then frees its memory. */
int bmfr_server_close_stream(bmfr_server* server, int stream_id);
int bmfr_server_stream_inputs(bmfr_server* server, int stream_id, bmfr_frame_inputs* inputs);
/* bmfr_batch_snapshot of an open stream once its submitted frames are done
 * (the stream stays open), and bmfr_batch_restore as an admitted stream:
 * moving a render stream between servers or GPUs between two frames. */
int bmfr_server_snapshot_stream(bmfr_server* server, int stream_id, void* dst, void* stream);
int bmfr_server_restore_stream(bmfr_server* server, const void* src, void* stream, int* stream_id);

/* Queues the stream's next frame.  io: the frame's device buffers (they and
 * the previous G-buffer pointers must stay valid until the request
 * completes); NULL uses the stream's input slots, which the caller fills for
 * one frame at a time (after the previous request completed).  io->result,
 * if not NULL, receives the output.  matrix/offset: host memory, copied.
 * Returns a request id. */
int bmfr_server_submit(bmfr_server* server, int stream_id, const bmfr_frame_io* io, const float* matrix,
                       const float* offset, uint64_t* request_id);
/* done = 1 once the request's step has finished on the GPU; latency from
 * submission to completion. */
int bmfr_server_poll(bmfr_server* server, uint64_t request_id, int* done, double* latency_ms);
/* Blocks until every submitted request has completed (or timeout_ms passes:
 * BMFR_E_TIMEOUT). */
int bmfr_server_drain(bmfr_server* server, double timeout_ms);
int bmfr_server_stats_get(bmfr_server* server, bmfr_server_stats* stats);
int bmfr_server_stats_reset(bmfr_server* server);
/* The batch underneath (read-only use while the server runs). */
bmfr_batch* bmfr_server_batch(bmfr_server* server);
/* bmfr_batch_set_tuning, serialised with the server's steps. */
int bmfr_server_set_tuning(bmfr_server* server, const bmfr_batch_tuning* tuning);

#ifdef __cplusplus
}
#endif
#endif /* BMFR_BATCH_H */
