// batch.cu — kernels of the many-stream engine (batched and served forms).
//
// The fused step: one frame of every participating stream, the streams'
// 32x32 blocks forming one global queue that a single persistent launch of
// the fused block kernel walks (accumulate + fit, and with the pixel pass
// off weighted sum + filtered accumulation, per block, fused_block.cuh),
// with the pixel pass a launch over the streams' pixel tiles for weighted
// sum + filtered accumulation, then one launch over their TAA tiles.  Both read the step's description from device memory,
// so one captured CUDA graph serves every step.  (The staged step runs the
// plan's kernels per stream, batch_host.cu.)
#include <type_traits>

#include "batch.cuh"
#include "fused_block.cuh"
#include "tma.cuh"

namespace bmfr {

namespace {

__device__ __forceinline__ int stream_of_block(const BatchStepDesc* __restrict__ d, int item) {
    int lo = 0, hi = d->n_streams - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (d->s[mid].block_start <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int stream_of_tile(const BatchStepDesc* __restrict__ d, int tile) {
    int lo = 0, hi = d->n_streams - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (d->s[mid].tile_start <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Prefetches into L2 the current-frame input rows of block `item` (normals,
// positions, colour and albedo of its 32 margin rows), by one warp.
__device__ void prefetch_block_inputs(const BatchStepDesc* __restrict__ d, int item) {
    const int lane = threadIdx.x & 31;
    const int s = stream_of_block(d, item);
    const BlockJob& j = d->s[s].job;
    const Geometry& g = j.g;
    const int b = item - d->s[s].block_start;
    const int bx = b % g.MWb, by = b / g.MWb;
    const int2 bo = c_block_offsets[j.a.frame & 15];
    const int row = mirror(by * kBlockEdge + lane - kBlockEdge / 2 + bo.y, g.H);
    int x0 = bx * kBlockEdge - kBlockEdge / 2 + bo.x, x1 = x0 + kBlockEdge;
    x0 = max(x0, 0);
    x1 = min(x1, g.W);
    if (x1 <= x0) return;
    // 16-byte aligned span covering pixels [x0, x1) of the row.
    const size_t first = ((size_t)row * g.W + x0) * 12;
    const size_t last = ((size_t)row * g.W + x1) * 12;
    const size_t a0 = first & ~(size_t)15, a1 = (last + 15) & ~(size_t)15;
    const uint32_t bytes = (uint32_t)(a1 - a0);
    const float* bufs[4] = {j.fb.cur_n, j.fb.cur_p, j.fb.noisy_in, j.fb.albedo};
#pragma unroll
    for (int k = 0; k < 4; ++k) prefetch_l2(reinterpret_cast<const char*>(bufs[k]) + a0, bytes);
}

}  // namespace

__global__ void __launch_bounds__(256) k_batch_noise(const BatchStepDesc* __restrict__ d) {
    const int n = d->n_streams * kNoiseTableFloats;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int s = e / kNoiseTableFloats, k = e % kNoiseTableFloats;
        const BlockJob& j = d->s[s].job;
        const_cast<float*>(j.fb.noise)[k] = noise_table_value(k, j.a.frame);
    }
}

// depth 0: blocks are taken from a global atomic queue; depth > 0: block
// blockIdx.x + k * gridDim.x, with the inputs of the CTA's next `depth`
// blocks prefetched into L2 while it fits the current one.
// PIXELS: see fused_block_body.
template <int METHOD, bool HALF_TMP, typename HistT, bool PIXELS>
__global__ void __launch_bounds__(256, (HALF_TMP && METHOD != kFitHouseholder32) ? 3 : 2)
    k_batch_blocks(const BatchStepDesc* __restrict__ d, int* __restrict__ counter, int depth) {
    __shared__ FitterSmem sm;
    __shared__ float w_s[kFeatures * 3], mm_s[kScaled * 2];
    __shared__ int item_s;
    const int nb = d->n_blocks;
    if (depth > 0) {
        if (threadIdx.x < 32)
            for (int k = 0; k < depth; ++k)
                if (blockIdx.x + k * (int)gridDim.x < nb) prefetch_block_inputs(d, blockIdx.x + k * gridDim.x);
        for (int item = blockIdx.x; item < nb; item += gridDim.x) {
            const int ahead = item + depth * (int)gridDim.x;
            if (threadIdx.x < 32 && ahead < nb) prefetch_block_inputs(d, ahead);
            const int s = stream_of_block(d, item);
            fused_block_body<METHOD, HALF_TMP, HistT, PIXELS>(d->s[s].job, item - d->s[s].block_start, sm, w_s,
                                                              mm_s);
            __syncthreads();
        }
    } else {
        for (;;) {
            if (threadIdx.x == 0) item_s = atomicAdd(counter, 1);
            __syncthreads();
            const int item = item_s;
            if (item >= nb) break;
            const int s = stream_of_block(d, item);
            fused_block_body<METHOD, HALF_TMP, HistT, PIXELS>(d->s[s].job, item - d->s[s].block_start, sm, w_s,
                                                              mm_s);
            __syncthreads();
        }
    }
}


// TAA tiles of 30 columns x 4R rows: four warps per CTA, R rows each
// (taa_strip).
template <int R, typename HistT>
__global__ void __launch_bounds__(128) k_batch_taa(const BatchStepDesc* __restrict__ d) {
    const int nt = d->n_tiles;
    for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
        const int s = stream_of_tile(d, tile);
        const BatchStreamJob& J = d->s[s];
        const int t = tile - J.tile_start;
        taa_strip<R, HistT>(J.job.g, J.job.a.frame, J.taa_alpha, (t % J.tiles_x) * 30,
                            (t / J.tiles_x) * 4 * R + (int)(threadIdx.x >> 5) * R, J.job.fb.prev_pix,
                            J.job.fb.tone_mapped, (const HistT*)J.result_prev, (HistT*)J.result_hist,
                            J.result_out);
    }
}

__device__ __forceinline__ int stream_of_px_tile(const BatchStepDesc* __restrict__ d, int tile) {
    int lo = 0, hi = d->n_streams - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (d->s[mid].px_tile_start <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The pixel pass: weighted_sum + accumulate_filtered_data over every
// stream's 32x8 pixel tiles (one thread per pixel, as the plan's kernel),
// the tone-mapped frame written for the TAA launch that follows.
template <typename HistT>
__global__ void __launch_bounds__(256) k_batch_wsacc(const BatchStepDesc* __restrict__ d) {
    const int nt = d->n_px_tiles;
    for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
        const int s = stream_of_px_tile(d, tile);
        const BatchStreamJob& J = d->s[s];
        const FusedBuffers& fb = J.job.fb;
        const Geometry& g = J.job.g;
        const int t = tile - J.px_tile_start;
        const int px = (t % J.px_tiles_x) * 32 + (threadIdx.x & 31), py = (t / J.px_tiles_x) * 8 + (threadIdx.x >> 5);
        if (px < g.W && py < g.H)
            wsacc_px<HistT>(g, J.job.a.frame, J.job.second_alpha, px, py, fb.weights, fb.mins_maxs, fb.cur_n,
                            fb.cur_p, nullptr, fb.prev_pix, fb.accept, fb.albedo, fb.tone_mapped, fb.cur_spp,
                            (const HistT*)fb.acc_prev, (HistT*)fb.acc_cur);
    }
}

cudaError_t launch_batch_noise(const BatchStepDesc* desc, int max_streams, cudaStream_t s) {
    const int grid = (max_streams * kNoiseTableFloats + 255) / 256;
    k_batch_noise<<<grid < 1184 ? grid : 1184, 256, 0, s>>>(desc);
    return cudaGetLastError();
}

template <int METHOD, bool HALF_TMP, typename HistT>
static cudaError_t launch_blocks_t(const BatchStepDesc* desc, int* counter, int depth, int grid, bool pixels,
                                   cudaStream_t s) {
    if (pixels) k_batch_blocks<METHOD, HALF_TMP, HistT, true><<<grid, kLocal, 0, s>>>(desc, counter, depth);
    else k_batch_blocks<METHOD, HALF_TMP, HistT, false><<<grid, kLocal, 0, s>>>(desc, counter, depth);
    return cudaGetLastError();
}

template <int METHOD, bool HALF_TMP, typename HistT>
static int occupancy_t() {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_blocks<METHOD, HALF_TMP, HistT, true>, kLocal,
                                                  0);
    return per_sm;
}

// The kernel instance for (qr, half_tmp, HistT) handed to F::run.
template <typename HistT, typename F>
static auto dispatch_blocks(int qr, bool half_tmp, F&& f) {
    if (!half_tmp) return f.template run<kFitReference, false, HistT>();
    if (qr == kFitCholQR2) return f.template run<kFitCholQR2, true, HistT>();
    if (qr == kFitHouseholder32) return f.template run<kFitHouseholder32, true, HistT>();
    return f.template run<kFitReference, true, HistT>();
}

struct LaunchBlocks {
    const BatchStepDesc* desc;
    int* counter;
    int depth, grid;
    bool pixels;
    cudaStream_t s;
    template <int M, bool H, typename T>
    cudaError_t run() const { return launch_blocks_t<M, H, T>(desc, counter, depth, grid, pixels, s); }
};

struct Occupancy {
    template <int M, bool H, typename T>
    int run() const { return occupancy_t<M, H, T>(); }
};

cudaError_t launch_batch_blocks(const BatchStepDesc* desc, int* counter, int qr, bool half_tmp,
                                bool half_history, int depth, int grid, bool pixels, cudaStream_t s) {
    const LaunchBlocks l{desc, counter, depth, grid, pixels, s};
    if (half_history) return dispatch_blocks<__half>(qr, half_tmp, l);
    return dispatch_blocks<float>(qr, half_tmp, l);
}

int batch_block_occupancy(int qr, bool half_tmp, bool half_history) {
    if (half_history) return dispatch_blocks<__half>(qr, half_tmp, Occupancy{});
    return dispatch_blocks<float>(qr, half_tmp, Occupancy{});
}


template <int R>
static cudaError_t launch_taa_t(const BatchStepDesc* desc, bool half_history, int sms, cudaStream_t s) {
    const int grid = sms * 16;
    if (half_history) k_batch_taa<R, __half><<<grid, 128, 0, s>>>(desc);
    else k_batch_taa<R, float><<<grid, 128, 0, s>>>(desc);
    return cudaGetLastError();
}

cudaError_t launch_batch_wsacc(const BatchStepDesc* desc, bool half_history, int sms, cudaStream_t s) {
    const int grid = sms * 32;
    if (half_history) k_batch_wsacc<__half><<<grid, 256, 0, s>>>(desc);
    else k_batch_wsacc<float><<<grid, 256, 0, s>>>(desc);
    return cudaGetLastError();
}

cudaError_t launch_batch_taa(const BatchStepDesc* desc, bool half_history, const BatchTuning& t, int sms,
                             cudaStream_t s) {
    if (t.tile_h == 8) return launch_taa_t<2>(desc, half_history, sms, s);
    if (t.tile_h == 16) return launch_taa_t<4>(desc, half_history, sms, s);
    if (t.tile_h == 64) return launch_taa_t<16>(desc, half_history, sms, s);
    return launch_taa_t<8>(desc, half_history, sms, s);
}

}  // namespace bmfr
