// fused_block.cuh — the per-block body of the frame pipeline's fused kernel
// (accumulate_noisy_data + fitter + weighted_sum + accumulate_filtered_data
// for one 32x32 block), shared by the single-stream kernel (fused.cu) and
// the many-stream block queue (batch.cu).
#pragma once

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
    t.set1(k, q, v);
}

// METHOD: FitMethod (the precision-form methods need HALF_TMP); with
// kFitReference and HALF_TMP the tile is binary16, rounded at every store as
// the reference rounds; HALF_TMP: features are rounded to binary16 as the
// reference's tmp_data stores them (bmfr.cl:471-475); HistT: element type of
// the colour histories.  PIXELS: phase 3 (weighted sum and filtered
// accumulation of the block's in-image pixels) runs here; without it the
// block ends at the fit and a per-pixel kernel runs them.  Block b of job j;
// ends with every thread past the fit's final barrier.
template <int METHOD, bool HALF_TMP, typename HistT, bool PIXELS = true>
__device__ __forceinline__ void fused_block_body(const BlockJob& j, int b, FitterSmem& sm, float* w_s,
                                                 float* mm_s) {
    constexpr bool ROUND = HALF_TMP && METHOD == kFitReference;
    const Geometry& g = j.g;
    const AccumArgs& a = j.a;
    const FusedBuffers& fb = j.fb;
    const float* __restrict__ cur_n = fb.cur_n;
    const float* __restrict__ prev_n = fb.prev_n;
    const float* __restrict__ cur_p = fb.cur_p;
    const float* __restrict__ prev_p = fb.prev_p;
    const float* __restrict__ noisy_in = fb.noisy_in;
    HistT* __restrict__ noisy_acc_cur = (HistT*)fb.noisy_acc_cur;
    const HistT* __restrict__ noisy_acc_prev = (const HistT*)fb.noisy_acc_prev;
    const uint8_t* __restrict__ prev_spp = fb.prev_spp;
    uint8_t* __restrict__ cur_spp = fb.cur_spp;
    float2* __restrict__ prev_pix = fb.prev_pix;
    uint8_t* __restrict__ accept = fb.accept;
    const float* __restrict__ albedo = fb.albedo;
    float* __restrict__ tone_mapped = fb.tone_mapped;
    const HistT* __restrict__ acc_prev = (const HistT*)fb.acc_prev;
    HistT* __restrict__ acc_cur = (HistT*)fb.acc_cur;
    const NoiseConst nc = j.nc;
    const float second_alpha = j.second_alpha;
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
        const AccumResult r = accumulate_core<HistT, true>(g, a, px, py, wp, nrm, cur, prev_n, prev_p, noisy_acc_prev,
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
    fit_block<ROUND, METHOD>(t, fb.noise, nc, sm, w_s, mm_s);
    if (threadIdx.x < kFeatures * 3) fb.weights[(size_t)b * kFeatures * 3 + threadIdx.x] = w_s[threadIdx.x];
    if (threadIdx.x < kScaled * 2) fb.mins_maxs[(size_t)b * kScaled * 2 + threadIdx.x] = mm_s[threadIdx.x];

    if constexpr (!PIXELS) return;
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

}  // namespace bmfr
