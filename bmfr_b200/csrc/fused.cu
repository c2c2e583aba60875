// fused.cu — the frame pipeline's block kernel: one 256-thread CTA per 32x32
// block runs accumulate_noisy_data for the block's 1024 margin pixels and the
// fitter (opencl/bmfr.cl:290-485, 490-700): the 13 feature columns go
// straight from the accumulation into the fitter's register tile, so
// tmp_data never reaches memory.  With `pixels` the same CTA then runs
// weighted_sum + accumulate_filtered_data for the block's in-image pixels
// (bmfr.cl:703-857) from the weights in shared memory; without it (the plan
// pipeline) those stages run as the plan's per-pixel kernel
// (k_weighted_sum_accumulate), which is not held to the fitter's three CTAs
// per SM.
//
// The margin grid is tiled exactly by the fitter's blocks, and a pixel's
// weights come from the block whose margin grid holds it unmirrored
// (bmfr.cl:718-722 inverts bmfr.cl:314-317).  Work-item id owns block pixels
// id + 256*q (q = 0..3) in every phase, so the owner of a pixel in the
// accumulation is the thread that later filters it and can keep its accept
// mask and spp in registers.
#include "fused_block.cuh"

namespace bmfr {

template <int METHOD, bool HALF_TMP, typename HistT, bool PIXELS>
__global__ void __launch_bounds__(256, (HALF_TMP && METHOD != kFitHouseholder32) ? 3 : 2) k_fused_block(BlockJob j) {
    await_previous_kernel();
    __shared__ FitterSmem sm;
    __shared__ float w_s[kFeatures * 3], mm_s[kScaled * 2];
    fused_block_body<METHOD, HALF_TMP, HistT, PIXELS>(j, blockIdx.x, sm, w_s, mm_s);
}

template <int METHOD, bool HALF_TMP, typename HistT>
static cudaError_t launch_fused_t(const Geometry& g, const AccumArgs& a, NoiseConst nc, float second_alpha,
                                  const FusedBuffers& fb, bool pixels, cudaStream_t s) {
    BlockJob j;
    j.g = g;
    j.a = a;
    j.nc = nc;
    j.second_alpha = second_alpha;
    j.fb = fb;
    if (pixels)
        return launch_chained(k_fused_block<METHOD, HALF_TMP, HistT, true>, dim3(g.blocks), dim3(kLocal), 0, s, j);
    return launch_chained(k_fused_block<METHOD, HALF_TMP, HistT, false>, dim3(g.blocks), dim3(kLocal), 0, s, j);
}

template <typename HistT>
static cudaError_t launch_fused_h(const Geometry& g, const AccumArgs& a, NoiseConst nc, float second_alpha,
                                  int qr, const FusedBuffers& fb, bool pixels, cudaStream_t s) {
    if (a.use_half == 0) return launch_fused_t<kFitReference, false, HistT>(g, a, nc, second_alpha, fb, pixels, s);
    if (qr == kFitCholQR2) return launch_fused_t<kFitCholQR2, true, HistT>(g, a, nc, second_alpha, fb, pixels, s);
    if (qr == kFitHouseholder32)
        return launch_fused_t<kFitHouseholder32, true, HistT>(g, a, nc, second_alpha, fb, pixels, s);
    return launch_fused_t<kFitReference, true, HistT>(g, a, nc, second_alpha, fb, pixels, s);
}

cudaError_t launch_fused_block(const Geometry& g, const AccumArgs& a, NoiseConst nc, float second_alpha,
                               int qr, bool half_history, const FusedBuffers& fb, bool pixels, cudaStream_t s) {
    if (half_history) return launch_fused_h<__half>(g, a, nc, second_alpha, qr, fb, pixels, s);
    return launch_fused_h<float>(g, a, nc, second_alpha, qr, fb, pixels, s);
}

}  // namespace bmfr
