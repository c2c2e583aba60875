// fused.cu — the frame pipeline's block kernel: one 256-thread CTA per 32x32
// block runs accumulate_noisy_data for the block's 1024 margin pixels, the
// fitter, and weighted_sum + accumulate_filtered_data for the block's
// in-image pixels (opencl/bmfr.cl:290-485, 490-700, 703-857).
//
// The margin grid is tiled exactly by the fitter's blocks, and a pixel's
// weights come from the block whose margin grid holds it unmirrored
// (bmfr.cl:718-722 inverts bmfr.cl:314-317), so every stage of the three
// stays inside one CTA: the 13 feature columns go straight from the
// accumulation into the fitter's register tile (tmp_data never reaches
// memory), and the weights stay in shared memory.  Only TAA, which reads a
// 3x3 neighbourhood across blocks, runs as a second kernel.
//
// Work-item id owns block pixels id + 256*q (q = 0..3) in all three phases,
// so the owner of a pixel in the accumulation is the thread that later
// filters it and can keep its accept mask and spp in registers.
#include "fused_block.cuh"

namespace bmfr {

template <int METHOD, bool HALF_TMP, typename HistT>
__global__ void __launch_bounds__(256, (HALF_TMP && METHOD != kFitHouseholder32) ? 3 : 2) k_fused_block(BlockJob j) {
    __shared__ FitterSmem sm;
    __shared__ float w_s[kFeatures * 3], mm_s[kScaled * 2];
    fused_block_body<METHOD, HALF_TMP, HistT>(j, blockIdx.x, sm, w_s, mm_s);
}

template <int METHOD, bool HALF_TMP, typename HistT>
static cudaError_t launch_fused_t(const Geometry& g, const AccumArgs& a, NoiseConst nc, float second_alpha,
                                  const FusedBuffers& fb, cudaStream_t s) {
    BlockJob j;
    j.g = g;
    j.a = a;
    j.nc = nc;
    j.second_alpha = second_alpha;
    j.fb = fb;
    k_fused_block<METHOD, HALF_TMP, HistT><<<g.blocks, kLocal, 0, s>>>(j);
    return cudaGetLastError();
}

template <typename HistT>
static cudaError_t launch_fused_h(const Geometry& g, const AccumArgs& a, NoiseConst nc, float second_alpha,
                                  int qr, const FusedBuffers& fb, cudaStream_t s) {
    if (a.use_half == 0) return launch_fused_t<kFitReference, false, HistT>(g, a, nc, second_alpha, fb, s);
    if (qr == kFitCholQR2) return launch_fused_t<kFitCholQR2, true, HistT>(g, a, nc, second_alpha, fb, s);
    if (qr == kFitHouseholder32) return launch_fused_t<kFitHouseholder32, true, HistT>(g, a, nc, second_alpha, fb, s);
    return launch_fused_t<kFitReference, true, HistT>(g, a, nc, second_alpha, fb, s);
}

cudaError_t launch_fused_block(const Geometry& g, const AccumArgs& a, NoiseConst nc, float second_alpha,
                               int qr, bool half_history, const FusedBuffers& fb, cudaStream_t s) {
    if (half_history) return launch_fused_h<__half>(g, a, nc, second_alpha, qr, fb, s);
    return launch_fused_h<float>(g, a, nc, second_alpha, qr, fb, s);
}

}  // namespace bmfr
