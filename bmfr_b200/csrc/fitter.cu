// fitter.cu — standalone fitter kernel (opencl/bmfr.cl:490-700).
//
// Persistent CTAs of 256 threads, as many as fit on the SMs.  Each CTA walks
// blocks b = blockIdx.x, + gridDim.x, ...: the block's 13 x 1024 tmp_data
// values arrive by one bulk TMA copy (contiguous 26 KB, no tensor map
// needed) into shared memory, move to registers, and the copy of the CTA's
// next block is issued at once so that it overlaps the fit.
//
// The feature-noise table of the frame is either formed by each CTA in its
// shared memory (the drop-in entry point: no scratch memory, so calls on
// different streams never share state) or read from a table that an earlier
// kernel of the frame pipeline wrote to global memory (smaller CTAs, more of
// them per SM).
#include <mutex>
#include <type_traits>

#include "fit_block.cuh"
#include "kernels.h"
#include "tma.cuh"

namespace bmfr {

template <bool HALF_TMP, bool NOISE_GLOBAL>
struct FitterShared {
    using TmpT = typename std::conditional<HALF_TMP, __half, float>::type;
    alignas(128) TmpT tile[kBuffers * kBlockPixels];
    FitterSmem sm;
    alignas(8) uint64_t bar;
    float noise[NOISE_GLOBAL ? 1 : kNoiseTableFloats];
};

// METHOD (FitMethod): kFitReference rounds like the reference (a binary16
// tile when tmp_data is binary16); the precision-form methods need binary16
// tmp_data and work on a float tile.
template <bool HALF_TMP, int METHOD, bool NOISE_GLOBAL>
__global__ void __launch_bounds__(256, (HALF_TMP && METHOD != kFitHouseholder32) ? 3 : 2)
    k_fitter(int nblocks, int frame, NoiseConst nc, const void* __restrict__ tmp, float* __restrict__ weights,
             float* __restrict__ mins_maxs, const float* __restrict__ noise_g, int* __restrict__ status) {
    using Shared = FitterShared<HALF_TMP, NOISE_GLOBAL>;
    using TmpT = typename Shared::TmpT;
    constexpr bool ROUND = HALF_TMP && METHOD == kFitReference;
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
    if (!NOISE_GLOBAL) fill_noise_table(S.noise, frame);
    const float* noise = NOISE_GLOBAL ? noise_g : S.noise;
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
                    if constexpr (HALF_TMP) t.set1(k, q, __half2float(col[q * kLocal]));
                    else t.set1(k, q, col[q * kLocal]);
                }
            }
        }
        __syncthreads();   // the buffer is free again
        const int next = b + gridDim.x;
        if (threadIdx.x == 0 && next < nblocks) {
            mbar_arrive_expect_tx(&S.bar, kTileBytes);
            bulk_copy_g2s(S.tile, src + (size_t)next * kTileBytes, kTileBytes, &S.bar);
        }
        fit_block<ROUND, METHOD>(t, noise, nc, S.sm, weights + (size_t)b * kFeatures * 3,
                                 mins_maxs + (size_t)b * kScaled * 2);
    }
}

// The frame's noise table in global memory (kNoiseTableFloats floats).
__global__ void __launch_bounds__(256) k_noise_table(int frame, float* __restrict__ table) {
    const int e = blockIdx.x * kLocal + threadIdx.x;
    if (e < kNoiseTableFloats) table[e] = noise_table_value(e, frame);
}

cudaError_t launch_noise_table(int frame, float* table, cudaStream_t s) {
    k_noise_table<<<kNoiseTableFloats / kLocal, kLocal, 0, s>>>(frame, table);
    return cudaGetLastError();
}

template <bool HALF_TMP, int METHOD, bool NOISE_GLOBAL>
static cudaError_t launch_fitter_t(int nblocks, int frame, NoiseConst nc, const void* tmp, float* weights,
                                   float* mins_maxs, const float* noise, int* status, cudaStream_t s) {
    auto kern = k_fitter<HALF_TMP, METHOD, NOISE_GLOBAL>;
    const int smem = (int)sizeof(FitterShared<HALF_TMP, NOISE_GLOBAL>);
    static int grid_cap[64] = {0};   // per device
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (grid_cap[dev] == 0) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
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
    kern<<<grid, kLocal, smem, s>>>(nblocks, frame, nc, tmp, weights, mins_maxs, noise, status);
    return cudaGetLastError();
}

cudaError_t launch_fitter(const Geometry& g, int frame, NoiseConst nc, const void* tmp, bool half_tmp,
                          int qr, float* weights, float* mins_maxs, const float* noise_table, int* status,
                          cudaStream_t s) {
    const int n = g.blocks;
    // The precision-form methods apply to binary16 tmp_data; float tmp_data
    // always takes the reference's arithmetic.
    const int method = half_tmp ? qr : kFitReference;
    if (noise_table) {
        if (!half_tmp)
            return launch_fitter_t<false, kFitReference, true>(n, frame, nc, tmp, weights, mins_maxs, noise_table,
                                                               status, s);
        if (method == kFitCholQR2)
            return launch_fitter_t<true, kFitCholQR2, true>(n, frame, nc, tmp, weights, mins_maxs, noise_table,
                                                            status, s);
        if (method == kFitHouseholder32)
            return launch_fitter_t<true, kFitHouseholder32, true>(n, frame, nc, tmp, weights, mins_maxs,
                                                                  noise_table, status, s);
        return launch_fitter_t<true, kFitReference, true>(n, frame, nc, tmp, weights, mins_maxs, noise_table,
                                                          status, s);
    }
    if (!half_tmp)
        return launch_fitter_t<false, kFitReference, false>(n, frame, nc, tmp, weights, mins_maxs, nullptr, status,
                                                            s);
    if (method == kFitCholQR2)
        return launch_fitter_t<true, kFitCholQR2, false>(n, frame, nc, tmp, weights, mins_maxs, nullptr, status, s);
    if (method == kFitHouseholder32)
        return launch_fitter_t<true, kFitHouseholder32, false>(n, frame, nc, tmp, weights, mins_maxs, nullptr,
                                                               status, s);
    return launch_fitter_t<true, kFitReference, false>(n, frame, nc, tmp, weights, mins_maxs, nullptr, status, s);
}

// ---------------------------------------------------------------------------
// Scratch in a static device array, for callers that cannot allocate.
//
// The fitter's scratch is the frame's noise table (kNoiseTableFloats floats)
// plus the bounded-wait status word.  Both live here in one file-scope device
// array, so launch_fitter_static needs no cudaMalloc.  The table does not
// grow with the image: this fixed size serves every image size a plan
// accepts.  In host code g_fitter_scratch only names the symbol; the device
// address comes from cudaGetSymbolAddress, taken once per device with that
// device current.
constexpr size_t kStaticStatusOffset = kNoiseTableBytes;             // 36,864
constexpr size_t kStaticScratchBytes = kStaticStatusOffset + 256;    // table + status word
static __device__ __align__(256) unsigned char g_fitter_scratch[kStaticScratchBytes];

static std::mutex g_scratch_mutex;
static void* g_scratch_address[64] = {nullptr};

static cudaError_t static_scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_address[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_fitter_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_address[dev] = p;
    }
    *out = g_scratch_address[dev];
    return cudaSuccess;
}

cudaError_t launch_fitter_static(const Geometry& g, int frame, NoiseConst nc, const void* tmp, bool half_tmp,
                                 int qr, float* weights, float* mins_maxs, cudaStream_t s) {
    void* base = nullptr;
    cudaError_t e = static_scratch_address(&base);
    if (e != cudaSuccess) return e;
    float* table = static_cast<float*>(base);
    int* status = reinterpret_cast<int*>(static_cast<unsigned char*>(base) + kStaticStatusOffset);
    e = cudaMemsetAsync(status, 0, sizeof(int), s);   // the array keeps the last call's contents
    if (e != cudaSuccess) return e;
    e = launch_noise_table(frame, table, s);
    if (e != cudaSuccess) return e;
    return launch_fitter(g, frame, nc, tmp, half_tmp, qr, weights, mins_maxs, table, status, s);
}

}  // namespace bmfr
