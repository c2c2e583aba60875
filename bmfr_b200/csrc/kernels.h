// kernels.h — host-side launchers of the sm_100a kernels (internal).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <utility>

#include "common.cuh"

namespace bmfr {

// Launches `kern` with programmatic stream serialization: its launch is
// processed while the previous kernel in the stream drains, and the kernel
// begins with await_previous_kernel() (common.cuh), so the stream's ordering
// is unchanged.  Measured on a 1280x720 frame of the plan pipeline: 164.8
// against 174.7 us with plain launches.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_chained(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                  Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// noisy_out/prev_noisy: the accumulated-colour history, float or (with
// half_history) binary16; noisy_in == noisy_out runs the in-place form.
cudaError_t launch_accumulate_noisy(const Geometry& g, const AccumArgs& a, float2* prev_pix, uint8_t* accept,
                                    const float* cur_n, const float* prev_n, const float* cur_p,
                                    const float* prev_p, const float* noisy_in, void* noisy_out,
                                    const void* prev_noisy, bool half_history, const uint8_t* prev_spp,
                                    uint8_t* cur_spp, void* tmp, cudaStream_t s);
// The fitter in double precision (precision form's reference).
cudaError_t launch_fitter_fp64(const Geometry& g, int frame, double noise_amount, const void* tmp, bool half_tmp,
                               double* weights, float* mins_maxs, cudaStream_t s);

// status: device word that receives a nonzero code if a bounded wait ran out.
// noise_table: the frame's table from launch_noise_table, or null to have
// every CTA form it in shared memory.  qr: bmfr_params.fp32_qr (0 the
// reference's arithmetic, 1 CholeskyQR2, 2 Householder in FP32).
cudaError_t launch_fitter(const Geometry& g, int frame, NoiseConst nc, const void* tmp, bool half_tmp,
                          int qr, float* weights, float* mins_maxs, const float* noise_table, int* status,
                          cudaStream_t s);
cudaError_t launch_noise_table(int frame, float* table, cudaStream_t s);
// One CTA waits, with the fitter's bounded wait limited to limit_ns, on a
// barrier that nothing completes, and records kDevTimeout in `status` when
// the limit runs out: the failure path of the bounded waits, without a fault.
cudaError_t launch_bounded_wait_probe(int* status, unsigned long long limit_ns, cudaStream_t s);
// The fitter with its scratch in a static device array (no allocation).
cudaError_t launch_fitter_static(const Geometry& g, int frame, NoiseConst nc, const void* tmp, bool half_tmp,
                                 int qr, float* weights, float* mins_maxs, cudaStream_t s);
// Device address of that array's bounded-wait status word (set-up on first
// use per device, ordered on `s`).
cudaError_t static_fitter_status(int** status, cudaStream_t s);
constexpr size_t kNoiseTableBytes = 9 * 4 * 256 * sizeof(float);

cudaError_t launch_weighted_sum(const Geometry& g, int frame, const float* weights, const float* mins_maxs,
                                float* out, const float* cur_n, const float* cur_p, cudaStream_t s);

cudaError_t launch_accumulate_filtered(const Geometry& g, int frame, float second_alpha, const float* filtered,
                                       const float2* prev_pix, const uint8_t* accept, const float* albedo,
                                       float* tone_mapped, const uint8_t* cur_spp, const float* acc_prev,
                                       float* acc_cur, cudaStream_t s);

cudaError_t launch_weighted_sum_accumulate(const Geometry& g, int frame, float second_alpha,
                                           const float* weights, const float* mins_maxs, const float* cur_n,
                                           const float* cur_p, float* filtered, const float2* prev_pix,
                                           const uint8_t* accept, const float* albedo, float* tone_mapped,
                                           const uint8_t* cur_spp, const void* acc_prev, void* acc_cur,
                                           bool half_history, cudaStream_t s);

cudaError_t launch_taa(const Geometry& g, int frame, float taa_alpha, const float2* prev_pix,
                       const float* new_frame, void* result, const void* prev_frame, float* result_f32,
                       bool half_history, cudaStream_t s);

// Buffers of the fused block kernel (accumulate + fit + weighted sum +
// filtered accumulation).  The four colour histories are float or binary16
// per the launch's half_history.
struct FusedBuffers {
    const float *cur_n, *prev_n, *cur_p, *prev_p, *noisy_in, *albedo;
    void* noisy_acc_cur;
    const void* noisy_acc_prev;
    const uint8_t* prev_spp;
    uint8_t* cur_spp;
    float2* prev_pix;
    uint8_t* accept;
    float* tone_mapped;
    const void* acc_prev;
    void* acc_cur;
    float *weights, *mins_maxs;
    const float* noise;   // the frame's noise table (launch_noise_table)
};

// Everything one 32x32 block of one stream needs in the fused block kernel.
struct BlockJob {
    Geometry g;
    AccumArgs a;
    NoiseConst nc;
    float second_alpha;
    FusedBuffers fb;
};

// pixels: the block kernel also runs weighted sum + filtered accumulation of
// the block's in-image pixels (tone-mapped frame written for a TAA launch).
cudaError_t launch_fused_block(const Geometry& g, const AccumArgs& a, NoiseConst nc, float second_alpha,
                               int qr, bool half_history, const FusedBuffers& fb, bool pixels, cudaStream_t s);

// NOISE_AMOUNT * 2 split into hi + lo floats, and the fitter's -0.0f.
inline NoiseConst make_noise_const(double noise_amount) {
    const double c = noise_amount * 2.0;
    NoiseConst n;
    n.hi = (float)c;
    n.lo = (float)(c - (double)n.hi);
    n.neg_zero = -0.0f;
    return n;
}

}  // namespace bmfr
