// fitter.cu — standalone fitter kernel (opencl/bmfr.cl:490-700): one
// 256-thread CTA per 32x32 block reads the block's 13 x 1024 tmp_data values
// once into registers and runs fit_block (fit_block.cuh).
#include "fit_block.cuh"
#include "kernels.h"

namespace bmfr {

template <bool HALF_TMP, bool ROUND>
__global__ void __launch_bounds__(256, 2) k_fitter(int frame, NoiseConst nc, const void* __restrict__ tmp,
                                                   float* __restrict__ weights, float* __restrict__ mins_maxs) {
    __shared__ FitterSmem sm;
    const int b = blockIdx.x;
    const int id = work_item_id();
    const size_t base = (size_t)b * kBuffers * kBlockPixels + id;
    float t[kBuffers][4];
#pragma unroll
    for (int k = 0; k < kBuffers; ++k)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const size_t i = base + (size_t)k * kBlockPixels + kLocal * q;
            t[k][q] = HALF_TMP ? __half2float(__ldg(reinterpret_cast<const __half*>(tmp) + i))
                               : __ldg(reinterpret_cast<const float*>(tmp) + i);
        }
    fit_block<ROUND>(t, frame, nc, sm, weights + (size_t)b * kFeatures * 3, mins_maxs + (size_t)b * kScaled * 2);
}

cudaError_t launch_fitter(const Geometry& g, int frame, NoiseConst nc, const void* tmp, bool half_tmp,
                          bool fp32_qr, float* weights, float* mins_maxs, cudaStream_t s) {
    const dim3 grid(g.blocks), block(kLocal);
    if (half_tmp && !fp32_qr)
        k_fitter<true, true><<<grid, block, 0, s>>>(frame, nc, tmp, weights, mins_maxs);
    else if (half_tmp)
        k_fitter<true, false><<<grid, block, 0, s>>>(frame, nc, tmp, weights, mins_maxs);
    else
        k_fitter<false, false><<<grid, block, 0, s>>>(frame, nc, tmp, weights, mins_maxs);
    return cudaGetLastError();
}

}  // namespace bmfr
