// fitter.cu — standalone fitter kernel (opencl/bmfr.cl:490-700).
//
// Persistent CTAs of 256 threads, as many as fit on the SMs.  Each CTA walks
// blocks b = blockIdx.x, + gridDim.x, ...: a block's 13 x 1024 tmp_data
// values arrive in shared memory by one TMA copy and move to registers, and
// the copy of a later block is issued at once so that it overlaps the fit.
//
// Binary16 tmp_data comes in as a 2-D tensor copy (rows of 64 halves, 208
// rows per block) with the 128-byte swizzle: the eight lanes of a warp that
// read one 16-byte chunk of a row meet three other lane groups at rows
// 64 halves apart, which without the swizzle fall in the same four banks
// (four-way conflicts on every load); the swizzle spreads them over 16
// banks.  With the frame's noise table in global memory the CTA keeps two
// tile buffers, so the copy of the block after next is in flight while the
// current one is fitted.  Float tmp_data uses a one-dimensional bulk copy.
//
// The feature-noise table of the frame is either formed by each CTA in its
// shared memory (the drop-in entry point: no scratch memory, so calls on
// different streams never share state) or read from a table that an earlier
// kernel of the frame pipeline wrote to global memory (smaller CTAs, more of
// them per SM).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <cstring>
#include <mutex>
#include <type_traits>

#include "fit_block.cuh"
#include "kernels.h"
#include "tma.cuh"

namespace bmfr {

constexpr int kTileRows = kBuffers * kBlockPixels / 64;   // 208 rows of 64 halves per block

template <bool HALF_TMP, bool NOISE_GLOBAL>
struct FitterShared {
    using TmpT = typename std::conditional<HALF_TMP, __half, float>::type;
    static constexpr int kStages = (HALF_TMP && NOISE_GLOBAL) ? 2 : 1;
    alignas(1024) TmpT tile[kStages][kBuffers * kBlockPixels];
    FitterSmem sm;
    alignas(8) uint64_t bar[kStages];
    float noise[NOISE_GLOBAL ? 1 : kNoiseTableFloats];
};

// Byte offset of half h of a block tile copied with the 128-byte swizzle:
// row h / 64, 16-byte chunk (h % 64) / 8 XOR the row's low three bits.
__device__ __forceinline__ uint32_t swizzled_half(uint32_t h) {
    const uint32_t r = h >> 6, c = h & 63u;
    return (r << 7) | ((((c >> 3) ^ r) & 7u) << 4) | ((c & 7u) << 1);
}

// METHOD (FitMethod): kFitReference rounds like the reference (a binary16
// tile when tmp_data is binary16); the precision-form methods need binary16
// tmp_data and work on a float tile.
template <bool HALF_TMP, int METHOD, bool NOISE_GLOBAL>
__global__ void __launch_bounds__(256, (HALF_TMP && METHOD != kFitHouseholder32) ? 3 : 2)
    k_fitter(int nblocks, int frame, NoiseConst nc, const void* __restrict__ tmp, const __grid_constant__ CUtensorMap tmap,
             float* __restrict__ weights, float* __restrict__ mins_maxs, const float* __restrict__ noise_g,
             int* __restrict__ status) {
    await_previous_kernel();
    using Shared = FitterShared<HALF_TMP, NOISE_GLOBAL>;
    using TmpT = typename Shared::TmpT;
    constexpr int kStages = Shared::kStages;
    constexpr bool ROUND = HALF_TMP && METHOD == kFitReference;
    extern __shared__ unsigned char smem_raw[];
    // The swizzled copy needs a 1024-byte aligned destination.
    Shared& S = *reinterpret_cast<Shared*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    constexpr uint32_t kTileBytes = kBuffers * kBlockPixels * sizeof(TmpT);
    const char* src = static_cast<const char*>(tmp);
    const int id = work_item_id();
    auto issue = [&](int stage, int blk) {
        mbar_arrive_expect_tx(&S.bar[stage], kTileBytes);
        if constexpr (HALF_TMP) tensor_copy_2d_g2s(S.tile[stage], &tmap, 0, blk * kTileRows, &S.bar[stage]);
        else bulk_copy_g2s(S.tile[stage], src + (size_t)blk * kTileBytes, kTileBytes, &S.bar[stage]);
    };

    if (threadIdx.x == 0) {
        for (int st = 0; st < kStages; ++st) mbar_init(&S.bar[st], 1);
        fence_barrier_init();
        S.sm.status = 0;
        for (int st = 0; st < kStages; ++st)
            if (blockIdx.x + st * (int)gridDim.x < nblocks) issue(st, blockIdx.x + st * gridDim.x);
    }
    if (!NOISE_GLOBAL) fill_noise_table(S.noise, frame);
    const float* noise = NOISE_GLOBAL ? noise_g : S.noise;
    __syncthreads();

    int it = 0;
    for (int b = blockIdx.x; b < nblocks; b += gridDim.x, ++it) {
        const int st = it % kStages;
        const uint32_t phase = (uint32_t)(it / kStages) & 1u;
        if (threadIdx.x == 0 && !mbar_wait_bounded(&S.bar[st], phase)) S.sm.status = kDevTimeout;
        __syncthreads();
        if (S.sm.status) {
            if (threadIdx.x == 0) {
                atomicExch(status, kDevTimeout);
                // let the copies in flight land
                for (int k = 0; k < kStages; ++k)
                    if (b + k * (int)gridDim.x < nblocks) mbar_wait_bounded(&S.bar[(it + k) % kStages], (uint32_t)((it + k) / kStages) & 1u);
            }
            return;
        }
        Tile<ROUND> t;
        const TmpT* tile = S.tile[st];
        // Row k*16 + 4q + id/64 of the tile holds (k, q); its swizzle XOR
        // (low three row bits) does not depend on k.
        uint32_t qoff[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) qoff[q] = swizzled_half((uint32_t)(q * kLocal + id));
#pragma unroll
        for (int k = 0; k < kBuffers; ++k) {
            if constexpr (HALF_TMP) {
                const unsigned char* base = reinterpret_cast<const unsigned char*>(tile) + k * kBlockPixels * 2;
                __half v[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) v[q] = *reinterpret_cast<const __half*>(base + qoff[q]);
                if constexpr (ROUND) {
                    t.h[k][0] = __halves2half2(v[0], v[1]);
                    t.h[k][1] = __halves2half2(v[2], v[3]);
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) t.set1(k, q, __half2float(v[q]));
                }
            } else {
                const TmpT* col = tile + k * kBlockPixels + id;
#pragma unroll
                for (int q = 0; q < 4; ++q) t.set1(k, q, col[q * kLocal]);
            }
        }
        __syncthreads();   // the buffer is free again
        const int next = b + kStages * (int)gridDim.x;
        if (threadIdx.x == 0 && next < nblocks) issue(st, next);
        fit_block<ROUND, METHOD>(t, noise, nc, S.sm, weights + (size_t)b * kFeatures * 3,
                                 mins_maxs + (size_t)b * kScaled * 2);
    }
}

// The frame's noise table in global memory (kNoiseTableFloats floats).
__global__ void __launch_bounds__(256) k_noise_table(int frame, float* __restrict__ table) {
    await_previous_kernel();
    const int e = blockIdx.x * kLocal + threadIdx.x;
    if (e < kNoiseTableFloats) table[e] = noise_table_value(e, frame);
}

cudaError_t launch_noise_table(int frame, float* table, cudaStream_t s) {
    return launch_chained(k_noise_table, dim3(kNoiseTableFloats / kLocal), dim3(kLocal), 0, s, frame, table);
}

// A barrier that no copy or thread ever completes: thread 0's bounded wait
// runs out after limit_ns and records the timeout as the fitter does.
__global__ void __launch_bounds__(32) k_bounded_wait_probe(int* __restrict__ status, unsigned long long limit_ns) {
    __shared__ alignas(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    __syncwarp();
    if (threadIdx.x == 0 && !mbar_wait_bounded(&bar, 0, limit_ns)) atomicExch(status, kDevTimeout);
}

cudaError_t launch_bounded_wait_probe(int* status, unsigned long long limit_ns, cudaStream_t s) {
    k_bounded_wait_probe<<<1, 32, 0, s>>>(status, limit_ns);
    return cudaGetLastError();
}

// cuTensorMapEncodeTiled from the driver, looked up once.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// binary16 tmp_data of `nblocks` blocks as rows of 64 halves; one box is
// one block (208 rows), swizzled by 128 bytes.
static cudaError_t encode_tmp_map(const void* tmp, int nblocks, CUtensorMap* map) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return cudaErrorNotSupported;
    const cuuint64_t dims[2] = {64, (cuuint64_t)nblocks * kTileRows};
    const cuuint64_t strides[1] = {128};
    const cuuint32_t box[2] = {64, (cuuint32_t)kTileRows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(tmp), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <bool HALF_TMP, int METHOD, bool NOISE_GLOBAL>
static cudaError_t launch_fitter_t(int nblocks, int frame, NoiseConst nc, const void* tmp, float* weights,
                                   float* mins_maxs, const float* noise, int* status, cudaStream_t s) {
    auto kern = k_fitter<HALF_TMP, METHOD, NOISE_GLOBAL>;
    const int smem = (int)sizeof(FitterShared<HALF_TMP, NOISE_GLOBAL>) + 1024;   // + alignment slack
    // Resident CTAs per device, found once per device and instantiation.
    // Threads that race on the first call compute the same value, so a
    // relaxed atomic store and load are enough.
    static std::atomic<int> grid_cap[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    int cap = grid_cap[dev].load(std::memory_order_relaxed);
    if (cap == 0) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kLocal, smem);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        cap = (per_sm > 0 ? per_sm : 1) * sms;
        grid_cap[dev].store(cap, std::memory_order_relaxed);
    }
    const int grid = nblocks < cap ? nblocks : cap;
    if (grid <= 0) return cudaSuccess;
    CUtensorMap map;
    std::memset(&map, 0, sizeof map);
    if (HALF_TMP) {
        e = encode_tmp_map(tmp, nblocks, &map);
        if (e != cudaSuccess) return e;
    }
    return launch_chained(kern, dim3(grid), dim3(kLocal), smem, s, nblocks, frame, nc, tmp, map, weights,
                          mins_maxs, noise, status);
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
// device current, when the status word is also cleared (on the caller's
// stream, ordered before the call's kernels).  From then on the word is
// sticky: a kernel that gives up a bounded wait sets it, and only
// static_fitter_status_clear (bmfr_fitter_noalloc_check) clears it.
constexpr size_t kStaticStatusOffset = kNoiseTableBytes;             // 36,864
constexpr size_t kStaticScratchBytes = kStaticStatusOffset + 256;    // table + status word
static __device__ __align__(256) unsigned char g_fitter_scratch[kStaticScratchBytes];

static std::mutex g_scratch_mutex;
static void* g_scratch_address[64] = {nullptr};

static cudaError_t static_scratch_address(void** out, cudaStream_t s) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_address[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_fitter_scratch);
        if (e != cudaSuccess) return e;
        e = cudaMemsetAsync(static_cast<unsigned char*>(p) + kStaticStatusOffset, 0, sizeof(int), s);
        if (e != cudaSuccess) return e;
        g_scratch_address[dev] = p;
    }
    *out = g_scratch_address[dev];
    return cudaSuccess;
}

cudaError_t static_fitter_status(int** status, cudaStream_t s) {
    void* base = nullptr;
    const cudaError_t e = static_scratch_address(&base, s);
    if (e != cudaSuccess) return e;
    *status = reinterpret_cast<int*>(static_cast<unsigned char*>(base) + kStaticStatusOffset);
    return cudaSuccess;
}

cudaError_t launch_fitter_static(const Geometry& g, int frame, NoiseConst nc, const void* tmp, bool half_tmp,
                                 int qr, float* weights, float* mins_maxs, cudaStream_t s) {
    void* base = nullptr;
    cudaError_t e = static_scratch_address(&base, s);
    if (e != cudaSuccess) return e;
    float* table = static_cast<float*>(base);
    int* status = reinterpret_cast<int*>(static_cast<unsigned char*>(base) + kStaticStatusOffset);
    e = launch_noise_table(frame, table, s);   // rewrites the table the last call left
    if (e != cudaSuccess) return e;
    return launch_fitter(g, frame, nc, tmp, half_tmp, qr, weights, mins_maxs, table, status, s);
}

}  // namespace bmfr
