// stages.cu — the four per-pixel stages of the BMFR pipeline on sm_100a:
// accumulate_noisy_data, weighted_sum, accumulate_filtered_data and taa
// (opencl/bmfr.cl:290-485, 703-758, 761-857, 860-974), plus the fused
// weighted_sum + accumulate_filtered_data kernel.
//
// All four are HBM-bound streaming kernels: one thread per pixel, 32x8
// threads per CTA so that each warp reads 32 consecutive interleaved float3
// pixels (384 contiguous bytes).  Their arithmetic keeps the reference's
// operation order exactly (the library is built with -fmad=false).
#include "kernels.h"
#include "pixel_ops.cuh"

namespace bmfr {

// ---------------------------------------------------------------------------
// accumulate_noisy_data
// ---------------------------------------------------------------------------

// MODE 0: every margin pixel computes from noisy_in (out-of-place);
// MODE 1: only in-image pixels, noisy_in == noisy_out (in-place, first pass);
// MODE 2: only mirrored margin pixels, taking the colour their in-image pixel
//         wrote in pass 1 (in-place, second pass).
// HistT: element type of the accumulated-colour history (noisy_out and
// prev_noisy); in-place modes use float.
template <int MODE, typename HistT>
__global__ void __launch_bounds__(256) k_accumulate_noisy(
    Geometry g, AccumArgs a, float2* __restrict__ prev_pix, uint8_t* __restrict__ accept,
    const float* __restrict__ cur_n, const float* __restrict__ prev_n,
    const float* __restrict__ cur_p, const float* __restrict__ prev_p,
    const float* noisy_in, HistT* noisy_out, const HistT* __restrict__ prev_noisy,
    const uint8_t* __restrict__ prev_spp, uint8_t* __restrict__ cur_spp, void* __restrict__ tmp) {
    await_previous_kernel();
    const int gx = blockIdx.x * 32 + threadIdx.x;
    const int gy = blockIdx.y * 8 + threadIdx.y;
    if constexpr (MODE == 0) {
        accumulate_margin_px<HistT>(g, a, gx, gy, prev_pix, accept, cur_n, prev_n, cur_p, prev_p, noisy_in, noisy_out,
                                    prev_noisy, prev_spp, cur_spp, tmp);
        return;
    }
    const int2 bo = c_block_offsets[a.frame & 15];
    const int pwx = gx - kBlockEdge / 2 + bo.x;
    const int pwy = gy - kBlockEdge / 2 + bo.y;
    const bool in_image = pwx >= 0 && pwx < g.W && pwy >= 0 && pwy < g.H;
    if (MODE == 1 && !in_image) return;
    if (MODE == 2 && in_image) return;
    const int px = mirror(pwx, g.W), py = mirror(pwy, g.H);
    const int lp = py * g.W + px;
    const float3 wp = load3(cur_p, lp);
    const float3 nrm = load3(cur_n, lp);
    if (MODE == 2) {
        store_tmp_row(g, tmp, a.use_half, gx, gy, wp, nrm, hist_load(noisy_out, lp));
        return;
    }
    const float3 cur = load3(noisy_in, lp);
    const AccumResult r = accumulate_core<HistT>(g, a, px, py, wp, nrm, cur, prev_n, prev_p, prev_noisy, prev_spp);
    store_tmp_row(g, tmp, a.use_half, gx, gy, wp, nrm, r.color);
    if (in_image) {   // bmfr.cl:442, 478-484
        cur_spp[lp] = r.spp;
        hist_store(noisy_out, lp, r.color);
        prev_pix[lp] = make_float2(r.ppx, r.ppy);
        accept[lp] = r.accept;
    }
}

// ---------------------------------------------------------------------------
// weighted_sum, accumulate_filtered_data, taa
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_weighted_sum(Geometry g, int frame,
                                                      const float* __restrict__ weights,
                                                      const float* __restrict__ mins_maxs,
                                                      float* __restrict__ out,
                                                      const float* __restrict__ cur_n,
                                                      const float* __restrict__ cur_p) {
    const int px = blockIdx.x * 32 + threadIdx.x, py = blockIdx.y * 8 + threadIdx.y;
    if (px >= g.W || py >= g.H) return;
    const int lp = py * g.W + px;
    const int gi = pixel_block(g, frame, px, py);
    store3(out, lp, weighted_sum_px(load3(cur_p, lp), load3(cur_n, lp), weights + (size_t)gi * kFeatures * 3,
                                    mins_maxs + (size_t)gi * kScaled * 2));
}

__global__ void __launch_bounds__(256) k_accumulate_filtered(
    Geometry g, int frame, float second_alpha, const float* __restrict__ filtered,
    const float2* __restrict__ prev_pix, const uint8_t* __restrict__ accept,
    const float* __restrict__ albedo, float* __restrict__ tone_mapped,
    const uint8_t* __restrict__ cur_spp, const float* __restrict__ acc_prev,
    float* __restrict__ acc_cur) {
    const int px = blockIdx.x * 32 + threadIdx.x, py = blockIdx.y * 8 + threadIdx.y;
    if (px >= g.W || py >= g.H) return;
    const int lp = py * g.W + px;
    float3 tm;
    const uint8_t acc = frame > 0 ? accept[lp] : 0;
    const float2 pp = acc ? prev_pix[lp] : make_float2(0.f, 0.f);
    const uint8_t spp = acc ? cur_spp[lp] : 1;
    const float3 a3 = accumulate_filtered_px(g, frame, lp, load3(filtered, lp), pp, acc, spp, second_alpha,
                                             acc_prev, load3(albedo, lp), &tm);
    store3(acc_cur, lp, a3);
    store3(tone_mapped, lp, tm);
}

// Fused weighted_sum + accumulate_filtered_data: both read the same pixel, so
// the filtered colour never goes to memory.  `filtered` may be null.
template <typename HistT>
__global__ void __launch_bounds__(256) k_weighted_sum_accumulate(
    Geometry g, int frame, float second_alpha, const float* __restrict__ weights,
    const float* __restrict__ mins_maxs, const float* __restrict__ cur_n,
    const float* __restrict__ cur_p, float* __restrict__ filtered,
    const float2* __restrict__ prev_pix, const uint8_t* __restrict__ accept,
    const float* __restrict__ albedo, float* __restrict__ tone_mapped,
    const uint8_t* __restrict__ cur_spp, const HistT* __restrict__ acc_prev,
    HistT* __restrict__ acc_cur) {
    await_previous_kernel();
    const int px = blockIdx.x * 32 + threadIdx.x, py = blockIdx.y * 8 + threadIdx.y;
    if (px >= g.W || py >= g.H) return;
    wsacc_px<HistT>(g, frame, second_alpha, px, py, weights, mins_maxs, cur_n, cur_p, filtered, prev_pix, accept,
                    albedo, tone_mapped, cur_spp, acc_prev, acc_cur);
}

// Rows per warp strip: 2 rows (4 rows loaded with the halo) keep more warps
// in flight than 8; measured at 1920x1080: 330.8 -> 321.3 us per frame.
constexpr int kTaaRows = 2;

template <typename HistT>
__global__ void __launch_bounds__(128) k_taa(Geometry g, int frame, float taa_alpha,
                                             const float2* __restrict__ prev_pix,
                                             const float* __restrict__ new_frame,
                                             HistT* __restrict__ result,
                                             const HistT* __restrict__ prev_frame,
                                             float* __restrict__ result_f32) {
    await_previous_kernel();
    taa_strip<kTaaRows, HistT>(g, frame, taa_alpha, blockIdx.x * 30, (blockIdx.y * 4 + (threadIdx.x >> 5)) * kTaaRows,
                               prev_pix, new_frame, prev_frame, result, result_f32);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

static dim3 margin_grid(const Geometry& g) { return dim3(g.MW / 32, g.MH / 8); }
static dim3 image_grid(const Geometry& g) { return dim3((g.W + 31) / 32, (g.H + 7) / 8); }
// TAA: 128-thread CTAs of four warps, each warp 30 columns x kTaaRows rows.
static dim3 taa_grid(const Geometry& g) { return dim3((g.W + 29) / 30, (g.H + 4 * kTaaRows - 1) / (4 * kTaaRows)); }

cudaError_t launch_accumulate_noisy(const Geometry& g, const AccumArgs& a, float2* prev_pix, uint8_t* accept,
                                    const float* cur_n, const float* prev_n, const float* cur_p,
                                    const float* prev_p, const float* noisy_in, void* noisy_out,
                                    const void* prev_noisy, bool half_history, const uint8_t* prev_spp,
                                    uint8_t* cur_spp, void* tmp, cudaStream_t s) {
    const dim3 grid = margin_grid(g), block(32, 8);
    if (half_history)
        return launch_chained(k_accumulate_noisy<0, __half>, grid, block, 0, s, g, a, prev_pix, accept, cur_n,
                              prev_n, cur_p, prev_p, noisy_in, (__half*)noisy_out, (const __half*)prev_noisy,
                              prev_spp, cur_spp, tmp);
    if (noisy_in == noisy_out) {
        float* io = (float*)noisy_out;
        const cudaError_t e = launch_chained(k_accumulate_noisy<1, float>, grid, block, 0, s, g, a, prev_pix, accept,
                                             cur_n, prev_n, cur_p, prev_p, noisy_in, io, (const float*)prev_noisy,
                                             prev_spp, cur_spp, tmp);
        if (e != cudaSuccess) return e;
        return launch_chained(k_accumulate_noisy<2, float>, grid, block, 0, s, g, a, prev_pix, accept, cur_n, prev_n,
                              cur_p, prev_p, noisy_in, io, (const float*)prev_noisy, prev_spp, cur_spp, tmp);
    }
    return launch_chained(k_accumulate_noisy<0, float>, grid, block, 0, s, g, a, prev_pix, accept, cur_n, prev_n,
                          cur_p, prev_p, noisy_in, (float*)noisy_out, (const float*)prev_noisy, prev_spp, cur_spp,
                          tmp);
}

cudaError_t launch_weighted_sum(const Geometry& g, int frame, const float* weights, const float* mins_maxs,
                                float* out, const float* cur_n, const float* cur_p, cudaStream_t s) {
    k_weighted_sum<<<image_grid(g), dim3(32, 8), 0, s>>>(g, frame, weights, mins_maxs, out, cur_n, cur_p);
    return cudaGetLastError();
}

cudaError_t launch_accumulate_filtered(const Geometry& g, int frame, float second_alpha, const float* filtered,
                                       const float2* prev_pix, const uint8_t* accept, const float* albedo,
                                       float* tone_mapped, const uint8_t* cur_spp, const float* acc_prev,
                                       float* acc_cur, cudaStream_t s) {
    k_accumulate_filtered<<<image_grid(g), dim3(32, 8), 0, s>>>(g, frame, second_alpha, filtered, prev_pix,
                                                                accept, albedo, tone_mapped, cur_spp,
                                                                acc_prev, acc_cur);
    return cudaGetLastError();
}

cudaError_t launch_weighted_sum_accumulate(const Geometry& g, int frame, float second_alpha,
                                           const float* weights, const float* mins_maxs, const float* cur_n,
                                           const float* cur_p, float* filtered, const float2* prev_pix,
                                           const uint8_t* accept, const float* albedo, float* tone_mapped,
                                           const uint8_t* cur_spp, const void* acc_prev, void* acc_cur,
                                           bool half_history, cudaStream_t s) {
    if (half_history)
        return launch_chained(k_weighted_sum_accumulate<__half>, image_grid(g), dim3(32, 8), 0, s, g, frame,
                              second_alpha, weights, mins_maxs, cur_n, cur_p, filtered, prev_pix, accept, albedo,
                              tone_mapped, cur_spp, (const __half*)acc_prev, (__half*)acc_cur);
    return launch_chained(k_weighted_sum_accumulate<float>, image_grid(g), dim3(32, 8), 0, s, g, frame, second_alpha,
                          weights, mins_maxs, cur_n, cur_p, filtered, prev_pix, accept, albedo, tone_mapped, cur_spp,
                          (const float*)acc_prev, (float*)acc_cur);
}

cudaError_t launch_taa(const Geometry& g, int frame, float taa_alpha, const float2* prev_pix,
                       const float* new_frame, void* result, const void* prev_frame, float* result_f32,
                       bool half_history, cudaStream_t s) {
    if (half_history)
        return launch_chained(k_taa<__half>, taa_grid(g), dim3(128), 0, s, g, frame, taa_alpha, prev_pix, new_frame,
                              (__half*)result, (const __half*)prev_frame, result_f32);
    return launch_chained(k_taa<float>, taa_grid(g), dim3(128), 0, s, g, frame, taa_alpha, prev_pix, new_frame,
                          (float*)result, (const float*)prev_frame, result_f32);
}

}  // namespace bmfr
