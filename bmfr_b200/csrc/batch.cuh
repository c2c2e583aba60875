// batch.cuh — device-side description of one step of the many-stream engine
// and its launchers (internal).
#pragma once

#include <cuda_runtime.h>

#include "kernels.h"

namespace bmfr {

constexpr int kBatchMaxStreams = 128;

// One stream taking part in a step.
struct BatchStreamJob {
    BlockJob job;              // geometry, per-frame arguments, buffers (this step's halves)
    int block_start;           // first block of this stream in the step's block queue
    int tile_start;            // first TAA tile of this stream
    int tiles_x;               // TAA tiles per image row (for the step's tile shape)
    int px_tile_start;         // first 32x8 pixel tile of this stream (the pixel pass)
    int px_tiles_x;            // pixel tiles per image row
    float taa_alpha;
    void* result_hist;         // TAA history written this frame (float or binary16)
    const void* result_prev;   // TAA history of the previous frame
    float* result_out;         // optional float copy of the output
    void* tmp;                 // the stream's tmp_data (staged step)
};

struct BatchStepDesc {
    int n_streams, n_blocks, n_tiles, tile_w, n_px_tiles;
    BatchStreamJob s[kBatchMaxStreams];
};

struct BatchTuning {
    int block_ctas_per_sm;   // persistent CTAs of the block kernel per SM
    int tile_w, tile_h;      // TAA CTA shape
    int staging_depth;       // blocks ahead whose inputs are prefetched into L2
    int pixel_pass;          // 1: weighted sum + filtered accumulation as a pass over pixel tiles
};

// The step's kernels read everything from `desc` (device memory), so one
// captured graph serves every step whatever streams take part.
cudaError_t launch_batch_noise(const BatchStepDesc* desc, int max_streams, cudaStream_t s);
// grid: persistent CTAs (from batch_block_occupancy and the tuning).
// qr: bmfr_params.fp32_qr (FitMethod).
// pixels: the block kernel also runs weighted sum + filtered accumulation.
cudaError_t launch_batch_blocks(const BatchStepDesc* desc, int* counter, int qr, bool half_tmp,
                                bool half_history, int depth, int grid, bool pixels, cudaStream_t s);
// The pixel pass: weighted sum + filtered accumulation over every stream's
// 32x8 pixel tiles, one thread per pixel.
cudaError_t launch_batch_wsacc(const BatchStepDesc* desc, bool half_history, int sms, cudaStream_t s);
cudaError_t launch_batch_taa(const BatchStepDesc* desc, bool half_history, const BatchTuning& t, int sms,
                             cudaStream_t s);
int batch_block_occupancy(int qr, bool half_tmp, bool half_history);


}  // namespace bmfr
