// fitter.cu — standalone fitter kernel (opencl/bmfr.cl:490-700).
//
// Persistent CTAs of 256 threads, as many as fit on the SMs (three per SM for
// the binary16 block).  Each CTA forms its frame's feature-noise table once,
// then walks blocks b = blockIdx.x, + gridDim.x, ...: the block's 13 x 1024
// tmp_data values arrive by one bulk TMA copy (contiguous 26 KB, no tensor
// map needed) into shared memory, move to registers, and the copy of the
// CTA's next block is issued at once so that it overlaps the fit.
#include "fit_block.cuh"
#include "kernels.h"
#include "tma.cuh"

namespace bmfr {

template <bool HALF_TMP>
struct FitterShared {
    using TmpT = typename std::conditional<HALF_TMP, __half, float>::type;
    NoiseTable nt;
    FitterSmem sm;
    alignas(128) TmpT tile[kBuffers * kBlockPixels];
    alignas(8) uint64_t bar;
};

template <bool HALF_TMP, bool ROUND>
__global__ void __launch_bounds__(256, (HALF_TMP && ROUND) ? 3 : 2)
    k_fitter(int nblocks, int frame, NoiseConst nc, const void* __restrict__ tmp, float* __restrict__ weights,
             float* __restrict__ mins_maxs, int* __restrict__ status) {
    using Shared = FitterShared<HALF_TMP>;
    using TmpT = typename Shared::TmpT;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    Shared& S = *reinterpret_cast<Shared*>(smem_raw);
    constexpr uint32_t kTileBytes = kBuffers * kBlockPixels * sizeof(TmpT);
    const char* src = static_cast<const char*>(tmp);
    const int id = work_item_id();

    int b = blockIdx.x;
    if (threadIdx.x == 0) {
        mbar_init(&S.bar, 1);
        fence_barrier_init();
        S.sm.status = 0;
        if (b < nblocks) {
            mbar_arrive_expect_tx(&S.bar, kTileBytes);
            bulk_copy_g2s(S.tile, src + (size_t)b * kTileBytes, kTileBytes, &S.bar);
        }
    }
    fill_noise_table(S.nt, frame);
    __syncthreads();

    uint32_t phase = 0;
    for (; b < nblocks; b += gridDim.x, phase ^= 1u) {
        if (threadIdx.x == 0 && !mbar_wait_bounded(&S.bar, phase)) S.sm.status = kDevTimeout;
        __syncthreads();
        if (S.sm.status) {
            if (threadIdx.x == 0) {
                atomicExch(status, kDevTimeout);
                mbar_wait_bounded(&S.bar, phase);   // let the copy in flight land
            }
            return;
        }
        Tile<ROUND> t;
#pragma unroll
        for (int k = 0; k < kBuffers; ++k) {
            const TmpT* col = S.tile + k * kBlockPixels + id;
            if constexpr (ROUND) {
                t.h[k][0] = __halves2half2(col[0], col[kLocal]);
                t.h[k][1] = __halves2half2(col[2 * kLocal], col[3 * kLocal]);
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if constexpr (HALF_TMP) t.f[k][q] = __half2float(col[q * kLocal]);
                    else t.f[k][q] = col[q * kLocal];
                }
            }
        }
        __syncthreads();   // the buffer is free again
        const int next = b + gridDim.x;
        if (threadIdx.x == 0 && next < nblocks) {
            mbar_arrive_expect_tx(&S.bar, kTileBytes);
            bulk_copy_g2s(S.tile, src + (size_t)next * kTileBytes, kTileBytes, &S.bar);
        }
        fit_block<ROUND>(t, S.nt, nc, S.sm, weights + (size_t)b * kFeatures * 3, mins_maxs + (size_t)b * kScaled * 2);
    }
}

template <bool HALF_TMP, bool ROUND>
static cudaError_t launch_fitter_t(int nblocks, int frame, NoiseConst nc, const void* tmp, float* weights,
                                   float* mins_maxs, int* status, cudaStream_t s) {
    auto kern = k_fitter<HALF_TMP, ROUND>;
    const int smem = (int)sizeof(FitterShared<HALF_TMP>);
    static int grid_cap[64] = {0};   // per device
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (grid_cap[dev] == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kLocal, smem);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        grid_cap[dev] = (per_sm > 0 ? per_sm : 1) * sms;
    }
    const int grid = nblocks < grid_cap[dev] ? nblocks : grid_cap[dev];
    if (grid <= 0) return cudaSuccess;
    kern<<<grid, kLocal, smem, s>>>(nblocks, frame, nc, tmp, weights, mins_maxs, status);
    return cudaGetLastError();
}

cudaError_t launch_fitter(const Geometry& g, int frame, NoiseConst nc, const void* tmp, bool half_tmp,
                          bool fp32_qr, float* weights, float* mins_maxs, int* status, cudaStream_t s) {
    if (half_tmp && !fp32_qr) return launch_fitter_t<true, true>(g.blocks, frame, nc, tmp, weights, mins_maxs, status, s);
    if (half_tmp) return launch_fitter_t<true, false>(g.blocks, frame, nc, tmp, weights, mins_maxs, status, s);
    return launch_fitter_t<false, false>(g.blocks, frame, nc, tmp, weights, mins_maxs, status, s);
}

}  // namespace bmfr
