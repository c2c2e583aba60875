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
#include "fit_block.cuh"
#include "kernels.h"
#include "pixel_ops.cuh"

namespace bmfr {

template <bool HALF>
__device__ __forceinline__ void tile_set1(Tile<HALF>& t, int k, int q, float v);
template <>
__device__ __forceinline__ void tile_set1(Tile<true>& t, int k, int q, float v) {
    const __half h = __float2half_rn(v);
    if (q & 1) t.h[k][q >> 1].y = h;
    else t.h[k][q >> 1].x = h;
}
template <>
__device__ __forceinline__ void tile_set1(Tile<false>& t, int k, int q, float v) {
    t.f[k][q] = v;
}

// ROUND: binary16 tile rounded at every store (reference arithmetic);
// HALF_TMP: features are rounded to binary16 as the reference's tmp_data
// stores them (bmfr.cl:471-475); HistT: element type of the colour histories.
template <bool ROUND, bool HALF_TMP, typename HistT>
__global__ void __launch_bounds__(256, 3) k_fused_block(
    Geometry g, AccumArgs a, NoiseConst nc, float second_alpha, const float* __restrict__ cur_n,
    const float* __restrict__ prev_n, const float* __restrict__ cur_p, const float* __restrict__ prev_p,
    const float* __restrict__ noisy_in, HistT* __restrict__ noisy_acc_cur,
    const HistT* __restrict__ noisy_acc_prev, const uint8_t* __restrict__ prev_spp,
    uint8_t* __restrict__ cur_spp, float2* __restrict__ prev_pix, uint8_t* __restrict__ accept,
    const float* __restrict__ albedo, float* __restrict__ tone_mapped, const HistT* __restrict__ acc_prev,
    HistT* __restrict__ acc_cur, float* __restrict__ weights, float* __restrict__ mins_maxs,
    const float* __restrict__ noise) {
    __shared__ FitterSmem sm;
    __shared__ float w_s[kFeatures * 3], mm_s[kScaled * 2];
    const int b = blockIdx.x;
    const int bx = b % g.MWb, by = b / g.MWb;
    const int id = work_item_id();
    const int2 bo = c_block_offsets[a.frame & 15];

    // Phase 1: accumulate_noisy_data of the block's margin pixels.
    Tile<ROUND> t;
    uint32_t owned = 0;            // bit q: pixel q is in the image (this is its owner)
    uint32_t as01 = 0, as23 = 0;   // accept | spp << 8 of pixels 0,1 and 2,3, 16 bits each
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int p = id + kLocal * q;
        const int gx = bx * kBlockEdge + (p & 31), gy = by * kBlockEdge + (p >> 5);
        const int pwx = gx - kBlockEdge / 2 + bo.x, pwy = gy - kBlockEdge / 2 + bo.y;
        const bool in_image = pwx >= 0 && pwx < g.W && pwy >= 0 && pwy < g.H;
        const int px = mirror(pwx, g.W), py = mirror(pwy, g.H);
        const int lp = py * g.W + px;
        const float3 wp = load3(cur_p, lp);
        const float3 nrm = load3(cur_n, lp);
        const float3 cur = load3(noisy_in, lp);
        const AccumResult r = accumulate_core<HistT>(g, a, px, py, wp, nrm, cur, prev_n, prev_p, noisy_acc_prev,
                                                     prev_spp);
        if (in_image) {   // bmfr.cl:442, 478-484
            owned |= 1u << q;
            const uint32_t v = (uint32_t)r.accept | ((uint32_t)r.spp << 8);
            if (q < 2) as01 |= v << (16 * q);
            else as23 |= v << (16 * (q - 2));
            cur_spp[lp] = r.spp;
            hist_store(noisy_acc_cur, lp, r.color);
            prev_pix[lp] = make_float2(r.ppx, r.ppy);
            accept[lp] = r.accept;
        }
        const float f[kBuffers] = {1.0f, nrm.x, nrm.y, nrm.z, wp.x, wp.y, wp.z, wp.x * wp.x, wp.y * wp.y,
                                   wp.z * wp.z, r.color.x, r.color.y, r.color.z};
#pragma unroll
        for (int k = 0; k < kBuffers; ++k) {
            float v = f[k];
            if (v != v) v = 0.0f;   // bmfr.cl:468-473
            if (HALF_TMP) v = fmaxf(fminf(v, 65504.0f), -65504.0f);
            if (HALF_TMP && !ROUND) v = round_half(v);
            tile_set1(t, k, q, v);
        }
    }

    // Phase 2: the fit; weights and min/max stay in shared memory.
    fit_block<ROUND, HALF_TMP && !ROUND>(t, noise, nc, sm, w_s, mm_s);
    if (threadIdx.x < kFeatures * 3) weights[(size_t)b * kFeatures * 3 + threadIdx.x] = w_s[threadIdx.x];
    if (threadIdx.x < kScaled * 2) mins_maxs[(size_t)b * kScaled * 2 + threadIdx.x] = mm_s[threadIdx.x];

    // Phase 3: weighted_sum and accumulate_filtered_data of the owned pixels.
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (!((owned >> q) & 1u)) continue;
        const int p = id + kLocal * q;
        const int px = bx * kBlockEdge + (p & 31) - kBlockEdge / 2 + bo.x;
        const int py = by * kBlockEdge + (p >> 5) - kBlockEdge / 2 + bo.y;
        const int lp = py * g.W + px;
        const uint32_t v = (q < 2 ? as01 >> (16 * q) : as23 >> (16 * (q - 2))) & 0xffffu;
        const uint8_t acc = (uint8_t)(v & 0xffu), spp = (uint8_t)(v >> 8);
        const float2 pp = acc ? prev_pix[lp] : make_float2(0.f, 0.f);
        const float3 filt = weighted_sum_px(load3(cur_p, lp), load3(cur_n, lp), w_s, mm_s);
        float3 tm;
        const float3 a3 = accumulate_filtered_px(g, a.frame, lp, filt, pp, acc, spp, second_alpha, acc_prev,
                                                 load3(albedo, lp), &tm);
        hist_store(acc_cur, lp, a3);
        store3(tone_mapped, lp, tm);
    }
}

template <bool ROUND, bool HALF_TMP, typename HistT>
static cudaError_t launch_fused_t(const Geometry& g, const AccumArgs& a, NoiseConst nc, float second_alpha,
                                  const FusedBuffers& fb, cudaStream_t s) {
    k_fused_block<ROUND, HALF_TMP, HistT><<<g.blocks, kLocal, 0, s>>>(
        g, a, nc, second_alpha, fb.cur_n, fb.prev_n, fb.cur_p, fb.prev_p, fb.noisy_in, (HistT*)fb.noisy_acc_cur,
        (const HistT*)fb.noisy_acc_prev, fb.prev_spp, fb.cur_spp, fb.prev_pix, fb.accept, fb.albedo,
        fb.tone_mapped, (const HistT*)fb.acc_prev, (HistT*)fb.acc_cur, fb.weights, fb.mins_maxs, fb.noise);
    return cudaGetLastError();
}

cudaError_t launch_fused_block(const Geometry& g, const AccumArgs& a, NoiseConst nc, float second_alpha,
                               bool fp32_qr, bool half_history, const FusedBuffers& fb, cudaStream_t s) {
    const bool half_tmp = a.use_half != 0;
    if (half_history) {
        if (half_tmp && !fp32_qr) return launch_fused_t<true, true, __half>(g, a, nc, second_alpha, fb, s);
        if (half_tmp) return launch_fused_t<false, true, __half>(g, a, nc, second_alpha, fb, s);
        return launch_fused_t<false, false, __half>(g, a, nc, second_alpha, fb, s);
    }
    if (half_tmp && !fp32_qr) return launch_fused_t<true, true, float>(g, a, nc, second_alpha, fb, s);
    if (half_tmp) return launch_fused_t<false, true, float>(g, a, nc, second_alpha, fb, s);
    return launch_fused_t<false, false, float>(g, a, nc, second_alpha, fb, s);
}

}  // namespace bmfr
