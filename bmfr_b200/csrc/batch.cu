// batch.cu — kernels of the many-stream engine (batched and served forms).
//
// One step denoises one frame of every participating stream.  The streams'
// 32x32 blocks form one global queue that a single persistent launch of the
// fused block kernel walks (accumulate + fit + weighted sum + filtered
// accumulation per block, fused_block.cuh); a second persistent launch walks
// the streams' TAA tiles.  Both read the step's description from device
// memory, so one captured CUDA graph serves every step.
#include "batch.cuh"
#include "fused_block.cuh"

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
template <bool ROUND, bool HALF_TMP, typename HistT>
__global__ void __launch_bounds__(256, ROUND ? 3 : 2)
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
            fused_block_body<ROUND, HALF_TMP, HistT>(d->s[s].job, item - d->s[s].block_start, sm, w_s, mm_s);
            __syncthreads();
        }
    } else {
        for (;;) {
            if (threadIdx.x == 0) item_s = atomicAdd(counter, 1);
            __syncthreads();
            const int item = item_s;
            if (item >= nb) break;
            const int s = stream_of_block(d, item);
            fused_block_body<ROUND, HALF_TMP, HistT>(d->s[s].job, item - d->s[s].block_start, sm, w_s, mm_s);
            __syncthreads();
        }
    }
}

template <int TW, int TH, typename HistT>
__global__ void __launch_bounds__(TW* TH) k_batch_taa(const BatchStepDesc* __restrict__ d) {
    const int nt = d->n_tiles;
    for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
        const int s = stream_of_tile(d, tile);
        const BatchStreamJob& J = d->s[s];
        const Geometry& g = J.job.g;
        const int t = tile - J.tile_start;
        const int px = (t % J.tiles_x) * TW + (int)(threadIdx.x % TW);
        const int py = (t / J.tiles_x) * TH + (int)(threadIdx.x / TW);
        if (px >= g.W || py >= g.H) continue;
        const int lp = py * g.W + px;
        const float3 r = taa_px(g, J.job.a.frame, J.taa_alpha, px, py, J.job.fb.prev_pix[lp], J.job.fb.tone_mapped,
                                (const HistT*)J.result_prev);
        hist_store((HistT*)J.result_hist, lp, r);
        if (J.result_out) store3(J.result_out, lp, r);
    }
}

cudaError_t launch_batch_noise(const BatchStepDesc* desc, int max_streams, cudaStream_t s) {
    const int grid = (max_streams * kNoiseTableFloats + 255) / 256;
    k_batch_noise<<<grid < 1184 ? grid : 1184, 256, 0, s>>>(desc);
    return cudaGetLastError();
}

template <bool ROUND, bool HALF_TMP, typename HistT>
static cudaError_t launch_blocks_t(const BatchStepDesc* desc, int* counter, int depth, int grid, cudaStream_t s) {
    k_batch_blocks<ROUND, HALF_TMP, HistT><<<grid, kLocal, 0, s>>>(desc, counter, depth);
    return cudaGetLastError();
}

cudaError_t launch_batch_blocks(const BatchStepDesc* desc, int* counter, bool fp32_qr, bool half_tmp,
                                bool half_history, int depth, int grid, cudaStream_t s) {
    if (half_history) {
        if (half_tmp && !fp32_qr) return launch_blocks_t<true, true, __half>(desc, counter, depth, grid, s);
        if (half_tmp) return launch_blocks_t<false, true, __half>(desc, counter, depth, grid, s);
        return launch_blocks_t<false, false, __half>(desc, counter, depth, grid, s);
    }
    if (half_tmp && !fp32_qr) return launch_blocks_t<true, true, float>(desc, counter, depth, grid, s);
    if (half_tmp) return launch_blocks_t<false, true, float>(desc, counter, depth, grid, s);
    return launch_blocks_t<false, false, float>(desc, counter, depth, grid, s);
}

int batch_block_occupancy(bool fp32_qr, bool half_tmp, bool half_history) {
    int per_sm = 0;
    if (half_history) {
        if (half_tmp && !fp32_qr)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_blocks<true, true, __half>, kLocal, 0);
        else if (half_tmp)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_blocks<false, true, __half>, kLocal, 0);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_blocks<false, false, __half>, kLocal, 0);
    } else {
        if (half_tmp && !fp32_qr)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_blocks<true, true, float>, kLocal, 0);
        else if (half_tmp)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_blocks<false, true, float>, kLocal, 0);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_blocks<false, false, float>, kLocal, 0);
    }
    return per_sm;
}

template <int TW, int TH>
static cudaError_t launch_taa_t(const BatchStepDesc* desc, bool half_history, int sms, cudaStream_t s) {
    const int grid = sms * (2048 / (TW * TH));
    if (half_history) k_batch_taa<TW, TH, __half><<<grid, TW * TH, 0, s>>>(desc);
    else k_batch_taa<TW, TH, float><<<grid, TW * TH, 0, s>>>(desc);
    return cudaGetLastError();
}

cudaError_t launch_batch_taa(const BatchStepDesc* desc, bool half_history, const BatchTuning& t, int sms,
                             cudaStream_t s) {
    if (t.tile_w == 32 && t.tile_h == 4) return launch_taa_t<32, 4>(desc, half_history, sms, s);
    if (t.tile_w == 64 && t.tile_h == 4) return launch_taa_t<64, 4>(desc, half_history, sms, s);
    if (t.tile_w == 16 && t.tile_h == 16) return launch_taa_t<16, 16>(desc, half_history, sms, s);
    return launch_taa_t<32, 8>(desc, half_history, sms, s);
}

}  // namespace bmfr
