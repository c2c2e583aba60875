// stages.cu — the four per-pixel stages of the BMFR pipeline on sm_100a:
// accumulate_noisy_data, weighted_sum, accumulate_filtered_data and taa
// (opencl/bmfr.cl:290-485, 703-758, 761-857, 860-974), plus the fused
// weighted_sum + accumulate_filtered_data kernel.
//
// All four are HBM-bound streaming kernels: one thread per pixel, 32x8
// threads per CTA so that each warp reads 32 consecutive interleaved float3
// pixels (384 contiguous bytes).  Their arithmetic keeps the reference's
// operation order exactly (the library is built with -fmad=false).
#include "common.cuh"
#include "kernels.h"

namespace bmfr {

// ---------------------------------------------------------------------------
// accumulate_noisy_data
// ---------------------------------------------------------------------------

struct AccumResult {
    float ppx, ppy;      // prev_frame_pixel_f
    float3 color;        // blended colour
    uint8_t accept;
    uint8_t spp;
};

// Reprojection, 4-tap history gather and blend of one pixel
// (bmfr.cl:319-445).  `cur` is the pixel's colour before blending.
__device__ __forceinline__ AccumResult accumulate_core(
    const Geometry& g, const AccumArgs& a, int px, int py, float3 wp, float3 nrm, float3 cur,
    const float* __restrict__ prev_n, const float* __restrict__ prev_p,
    const float* __restrict__ prev_noisy, const uint8_t* __restrict__ prev_spp) {
    AccumResult r;
    r.ppx = (float)px;
    r.ppy = (float)py;
    r.accept = 0;
    float alpha = 1.0f;
    float3 prev = make_float3(0.f, 0.f, 0.f);
    float sample_spp = 0.0f;
    if (a.frame > 0) {
        const float* m = a.m;
        float uvx = ((m[0] * wp.x + m[4] * wp.y) + m[8] * wp.z) + m[12] * 1.0f;
        float uvy = ((m[1] * wp.x + m[5] * wp.y) + m[9] * wp.z) + m[13] * 1.0f;
        const float w = ((m[3] * wp.x + m[7] * wp.y) + m[11] * wp.z) + m[15] * 1.0f;
        uvx = uvx / w;
        uvy = uvy / w;
        uvx = (uvx + 1.0f) / 2.0f;
        uvy = (uvy + 1.0f) / 2.0f;
        r.ppx = uvx * (float)g.W - a.off_x;
        r.ppy = uvy * (float)g.H - (1.0f - a.off_y);
        const int ix = floor_to_int(r.ppx), iy = floor_to_int(r.ppy);
        const float fx = r.ppx - (float)ix, fy = r.ppy - (float)iy;
        const float ofx = 1.0f - fx, ofy = 1.0f - fy;
        const float wts[4] = {ofx * ofy, fx * ofy, ofx * fy, fx * fy};
        float total = 0.0f;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int sx = ix + (i & 1), sy = iy + (i >> 1);
            if (sx >= 0 && sy >= 0 && sx < g.W && sy < g.H) {
                const int s = sy * g.W + sx;
                const float3 pp = load3(prev_p, s);
                const float dx = pp.x - wp.x, dy = pp.y - wp.y, dz = pp.z - wp.z;
                if ((dx * dx + dy * dy) + dz * dz < a.pos_lim2) {
                    const float3 pn = load3(prev_n, s);
                    const float ex = pn.x - nrm.x, ey = pn.y - nrm.y, ez = pn.z - nrm.z;
                    if ((ex * ex + ey * ey) + ez * ez < a.nrm_lim2) {
                        r.accept |= (uint8_t)(1 << i);
                        sample_spp = sample_spp + wts[i] * (float)prev_spp[s];
                        const float3 pc = load3(prev_noisy, s);
                        prev.x = prev.x + wts[i] * pc.x;
                        prev.y = prev.y + wts[i] * pc.y;
                        prev.z = prev.z + wts[i] * pc.z;
                        total = total + wts[i];
                    }
                }
            }
        }
        if (total > 0.0f) {
            prev.x = prev.x / total;
            prev.y = prev.y / total;
            prev.z = prev.z / total;
            sample_spp = sample_spp / total;
            alpha = 1.0f / (sample_spp + 1.0f);
            alpha = fmax_cl(alpha, a.blend_alpha);
        }
    }
    r.spp = 1;
    if (alpha < 1.0f) {
        if (sample_spp > 254.0f) {
            r.spp = 255;
        } else {
            float q = rintf(sample_spp);
            q = q < 0.f ? 0.f : (q > 255.f ? 255.f : q);
            r.spp = (uint8_t)((int)q + 1);
        }
    }
    const float om = 1.0f - alpha;
    r.color = make_float3(alpha * cur.x + om * prev.x, alpha * cur.y + om * prev.y,
                          alpha * cur.z + om * prev.z);
    return r;
}

// Writes the 13 feature/colour values of margin pixel (gx, gy) into the
// block-major tmp_data (bmfr.cl:448-476).
__device__ __forceinline__ void store_tmp_row(const Geometry& g, void* tmp, bool half_tmp, int gx,
                                              int gy, float3 wp, float3 nrm, float3 c) {
    const int xb = gx >> 5, yb = gy >> 5, xin = gx & 31, yin = gy & 31;
    const size_t base = (size_t)(yb * g.MWb + xb) * kBuffers * kBlockPixels + (size_t)(yin * 32 + xin);
    const float f[kBuffers] = {1.0f, nrm.x, nrm.y, nrm.z, wp.x, wp.y, wp.z,
                               wp.x * wp.x, wp.y * wp.y, wp.z * wp.z, c.x, c.y, c.z};
#pragma unroll
    for (int k = 0; k < kBuffers; ++k) store_feature(tmp, base + (size_t)k * kBlockPixels, f[k], half_tmp);
}

// MODE 0: every margin pixel computes from noisy_in (out-of-place);
// MODE 1: only in-image pixels, noisy_in == noisy_out (in-place, first pass);
// MODE 2: only mirrored margin pixels, taking the colour their in-image pixel
//         wrote in pass 1 (in-place, second pass).
template <int MODE>
__global__ void __launch_bounds__(256) k_accumulate_noisy(
    Geometry g, AccumArgs a, float2* __restrict__ prev_pix, uint8_t* __restrict__ accept,
    const float* __restrict__ cur_n, const float* __restrict__ prev_n,
    const float* __restrict__ cur_p, const float* __restrict__ prev_p,
    const float* noisy_in, float* noisy_out, const float* __restrict__ prev_noisy,
    const uint8_t* __restrict__ prev_spp, uint8_t* __restrict__ cur_spp, void* __restrict__ tmp) {
    const int gx = blockIdx.x * 32 + threadIdx.x;
    const int gy = blockIdx.y * 8 + threadIdx.y;
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
        store_tmp_row(g, tmp, a.use_half, gx, gy, wp, nrm, load3(noisy_out, lp));
        return;
    }
    const float3 cur = load3(noisy_in, lp);
    const AccumResult r = accumulate_core(g, a, px, py, wp, nrm, cur, prev_n, prev_p, prev_noisy, prev_spp);
    store_tmp_row(g, tmp, a.use_half, gx, gy, wp, nrm, r.color);
    if (in_image) {   // bmfr.cl:442, 478-484
        cur_spp[lp] = r.spp;
        store3(noisy_out, lp, r.color);
        prev_pix[lp] = make_float2(r.ppx, r.ppy);
        accept[lp] = r.accept;
    }
}

// ---------------------------------------------------------------------------
// weighted_sum, accumulate_filtered_data, taa
// ---------------------------------------------------------------------------

// weighted_sum body (bmfr.cl:712-750).
__device__ __forceinline__ float3 weighted_sum_px(const Geometry& g, int frame, int px, int py,
                                                  float3 wp, float3 n,
                                                  const float* __restrict__ weights,
                                                  const float* __restrict__ mins_maxs) {
    const int2 bo = c_block_offsets[frame & 15];
    const int opx = px + kBlockEdge / 2 - bo.x, opy = py + kBlockEdge / 2 - bo.y;
    const int gi = (opx / kBlockEdge) + (opy / kBlockEdge) * g.MWb;
    const float f[kFeatures] = {1.0f, n.x, n.y, n.z, wp.x, wp.y, wp.z, wp.x * wp.x, wp.y * wp.y, wp.z * wp.z};
    const float* w = weights + (size_t)gi * kFeatures * 3;
    const float* mm = mins_maxs + (size_t)gi * kScaled * 2;
    float3 c = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < kFeatures; ++k) {
        float v = f[k];
        if (k >= kNotScaled) v = scale(v, __ldg(mm + (k - kNotScaled) * 2), __ldg(mm + (k - kNotScaled) * 2 + 1));
        c.x = c.x + __ldg(w + 3 * k) * v;
        c.y = c.y + __ldg(w + 3 * k + 1) * v;
        c.z = c.z + __ldg(w + 3 * k + 2) * v;
    }
    c.x = c.x < 0.f ? 0.f : c.x;
    c.y = c.y < 0.f ? 0.f : c.y;
    c.z = c.z < 0.f ? 0.f : c.z;
    return c;
}

__global__ void __launch_bounds__(256) k_weighted_sum(Geometry g, int frame,
                                                      const float* __restrict__ weights,
                                                      const float* __restrict__ mins_maxs,
                                                      float* __restrict__ out,
                                                      const float* __restrict__ cur_n,
                                                      const float* __restrict__ cur_p) {
    const int px = blockIdx.x * 32 + threadIdx.x, py = blockIdx.y * 8 + threadIdx.y;
    if (px >= g.W || py >= g.H) return;
    const int lp = py * g.W + px;
    store3(out, lp, weighted_sum_px(g, frame, px, py, load3(cur_p, lp), load3(cur_n, lp), weights, mins_maxs));
}

// accumulate_filtered_data body (bmfr.cl:778-856); returns the accumulated
// colour and writes the tone-mapped one through `tm`.
template <typename HistT>
__device__ __forceinline__ float3 accumulate_filtered_px(const Geometry& g, int frame, int lp, float3 filt,
                                                         float2 pp, uint8_t acc, uint8_t spp,
                                                         float second_alpha, const HistT* __restrict__ acc_prev,
                                                         float3 albedo, float3* tm);

__device__ __forceinline__ float3 hist_load(const float* p, int i) { return load3(p, i); }
__device__ __forceinline__ float3 hist_load(const __half* p, int i) {
    return make_float3(__half2float(p[3 * i]), __half2float(p[3 * i + 1]), __half2float(p[3 * i + 2]));
}

// Tone map: clamp(powr(max(0, albedo * acc), 0.454545), 0, 1) (bmfr.cl:853-854).
__device__ __forceinline__ float tonemap1(float albedo, float acc) {
    const float x = fmax_cl(0.0f, albedo * acc);
    const float t = x > 0.0f ? powf(x, 0.454545f) : 0.0f;
    return fmin_cl(fmax_cl(t, 0.0f), 1.0f);
}

template <typename HistT>
__device__ __forceinline__ float3 accumulate_filtered_px(const Geometry& g, int frame, int lp, float3 filt,
                                                         float2 pp, uint8_t acc, uint8_t spp,
                                                         float second_alpha, const HistT* __restrict__ acc_prev,
                                                         float3 albedo, float3* tm) {
    float3 prev = make_float3(0.f, 0.f, 0.f);
    float alpha = 1.0f;
    if (frame > 0 && acc > 0) {
        const int ix = floor_to_int(pp.x), iy = floor_to_int(pp.y);
        const float fx = pp.x - (float)ix, fy = pp.y - (float)iy;
        const float ofx = 1.0f - fx, ofy = 1.0f - fy;
        const float wts[4] = {ofx * ofy, fx * ofy, ofx * fy, fx * fy};
        float total = 0.0f;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (acc & (1 << i)) {
                total = total + wts[i];
                const float3 c = hist_load(acc_prev, (iy + (i >> 1)) * g.W + ix + (i & 1));
                prev.x = prev.x + wts[i] * c.x;
                prev.y = prev.y + wts[i] * c.y;
                prev.z = prev.z + wts[i] * c.z;
            }
        }
        if (total > 0.0f) {
            alpha = 1.0f / (float)spp;
            alpha = fmax_cl(alpha, second_alpha);
            prev.x = prev.x / total;
            prev.y = prev.y / total;
            prev.z = prev.z / total;
        }
    }
    const float om = 1.0f - alpha;
    const float3 a3 = make_float3(alpha * filt.x + om * prev.x, alpha * filt.y + om * prev.y,
                                  alpha * filt.z + om * prev.z);
    *tm = make_float3(tonemap1(albedo.x, a3.x), tonemap1(albedo.y, a3.y), tonemap1(albedo.z, a3.z));
    return a3;
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
    const int px = blockIdx.x * 32 + threadIdx.x, py = blockIdx.y * 8 + threadIdx.y;
    if (px >= g.W || py >= g.H) return;
    const int lp = py * g.W + px;
    const float3 f = weighted_sum_px(g, frame, px, py, load3(cur_p, lp), load3(cur_n, lp), weights, mins_maxs);
    if (filtered) store3(filtered, lp, f);
    float3 tm;
    const uint8_t acc = frame > 0 ? accept[lp] : 0;
    const float2 pp = acc ? prev_pix[lp] : make_float2(0.f, 0.f);
    const uint8_t spp = acc ? cur_spp[lp] : 1;
    const float3 a3 = accumulate_filtered_px(g, frame, lp, f, pp, acc, spp, second_alpha, acc_prev,
                                             load3(albedo, lp), &tm);
    hist_store(acc_cur, lp, a3);
    store3(tone_mapped, lp, tm);
}

// taa body (bmfr.cl:873-973).
template <typename HistT>
__device__ __forceinline__ float3 taa_px(const Geometry& g, int frame, float taa_alpha, int px, int py,
                                         float2 pp, const float* __restrict__ new_frame,
                                         const HistT* __restrict__ prev_frame) {
    const int lp = py * g.W + px;
    const float3 mine = load3(new_frame, lp);
    const int ix = floor_to_int(pp.x), iy = floor_to_int(pp.y);
    if (frame == 0 || ix < -1 || iy < -1 || ix >= g.W || iy >= g.H) return mine;
    float mnb[3] = {INFINITY, INFINITY, INFINITY}, mnc[3] = {INFINITY, INFINITY, INFINITY};
    float mxb[3] = {-INFINITY, -INFINITY, -INFINITY}, mxc[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
    for (int y = -1; y < 2; ++y) {
#pragma unroll
        for (int x = -1; x < 2; ++x) {
            const int sx = px + x, sy = py + y;
            if (sx >= 0 && sy >= 0 && sx < g.W && sy < g.H) {
                const float3 s = (x == 0 && y == 0) ? mine : load3(new_frame, sy * g.W + sx);
                const float ycc[3] = {(s.x * 1.0f + s.y * 2.0f) + s.z * 1.0f,
                                      (s.x * 2.0f + s.y * 0.0f) + s.z * -2.0f,
                                      (s.x * -1.0f + s.y * 2.0f) + s.z * -1.0f};
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    if (x == 0 || y == 0) {
                        mnc[c] = fmin_cl(mnc[c], ycc[c]);
                        mxc[c] = fmax_cl(mxc[c], ycc[c]);
                    }
                    mnb[c] = fmin_cl(mnb[c], ycc[c]);
                    mxb[c] = fmax_cl(mxb[c], ycc[c]);
                }
            }
        }
    }
    float3 prev = make_float3(0.f, 0.f, 0.f);
    float total = 0.0f;
    const float fx = pp.x - (float)ix, fy = pp.y - (float)iy;
    const float ofx = 1.0f - fx, ofy = 1.0f - fy;
    auto tap = [&](int sx, int sy, float w) {
        const float3 s = hist_load(prev_frame, sy * g.W + sx);
        prev.x = prev.x + w * s.x;
        prev.y = prev.y + w * s.y;
        prev.z = prev.z + w * s.z;
        total = total + w;
    };
    if (iy >= 0) {
        if (ix >= 0) tap(ix, iy, ofx * ofy);
        if (ix < g.W - 1) tap(ix + 1, iy, fx * ofy);
    }
    if (iy < g.H - 1) {
        if (ix >= 0) tap(ix, iy + 1, ofx * fy);
        if (ix < g.W - 1) tap(ix + 1, iy + 1, fx * fy);
    }
    prev.x = prev.x / total;
    prev.y = prev.y / total;
    prev.z = prev.z / total;
    const float pyc[3] = {(prev.x * 1.0f + prev.y * 2.0f) + prev.z * 1.0f,
                          (prev.x * 2.0f + prev.y * 0.0f) + prev.z * -2.0f,
                          (prev.x * -1.0f + prev.y * 2.0f) + prev.z * -1.0f};
    float cl[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float lo = (mnb[c] + mnc[c]) / 2.0f;
        const float hi = (mxb[c] + mxc[c]) / 2.0f;
        cl[c] = fmin_cl(fmax_cl(pyc[c], lo), hi);
    }
    const float3 rgb = make_float3((cl[0] * 0.25f + cl[1] * 0.25f) + cl[2] * -0.25f,
                                   (cl[0] * 0.25f + cl[1] * 0.0f) + cl[2] * 0.25f,
                                   (cl[0] * 0.25f + cl[1] * -0.25f) + cl[2] * -0.25f);
    const float om = 1.0f - taa_alpha;
    return make_float3(taa_alpha * mine.x + om * rgb.x, taa_alpha * mine.y + om * rgb.y,
                       taa_alpha * mine.z + om * rgb.z);
}

template <typename HistT>
__global__ void __launch_bounds__(256) k_taa(Geometry g, int frame, float taa_alpha,
                                             const float2* __restrict__ prev_pix,
                                             const float* __restrict__ new_frame,
                                             HistT* __restrict__ result,
                                             const HistT* __restrict__ prev_frame,
                                             float* __restrict__ result_f32) {
    const int px = blockIdx.x * 32 + threadIdx.x, py = blockIdx.y * 8 + threadIdx.y;
    if (px >= g.W || py >= g.H) return;
    const int lp = py * g.W + px;
    const float3 r = taa_px(g, frame, taa_alpha, px, py, prev_pix[lp], new_frame, prev_frame);
    hist_store(result, lp, r);
    if (result_f32) store3(result_f32, lp, r);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

static dim3 margin_grid(const Geometry& g) { return dim3(g.MW / 32, g.MH / 8); }
static dim3 image_grid(const Geometry& g) { return dim3((g.W + 31) / 32, (g.H + 7) / 8); }

cudaError_t launch_accumulate_noisy(const Geometry& g, const AccumArgs& a, float2* prev_pix,
                                    uint8_t* accept, const float* cur_n, const float* prev_n,
                                    const float* cur_p, const float* prev_p, const float* noisy_in,
                                    float* noisy_out, const float* prev_noisy, const uint8_t* prev_spp,
                                    uint8_t* cur_spp, void* tmp, cudaStream_t s) {
    const dim3 block(32, 8);
    if (noisy_in == noisy_out) {
        k_accumulate_noisy<1><<<margin_grid(g), block, 0, s>>>(g, a, prev_pix, accept, cur_n, prev_n, cur_p,
                                                               prev_p, noisy_in, noisy_out, prev_noisy,
                                                               prev_spp, cur_spp, tmp);
        k_accumulate_noisy<2><<<margin_grid(g), block, 0, s>>>(g, a, prev_pix, accept, cur_n, prev_n, cur_p,
                                                               prev_p, noisy_in, noisy_out, prev_noisy,
                                                               prev_spp, cur_spp, tmp);
    } else {
        k_accumulate_noisy<0><<<margin_grid(g), block, 0, s>>>(g, a, prev_pix, accept, cur_n, prev_n, cur_p,
                                                               prev_p, noisy_in, noisy_out, prev_noisy,
                                                               prev_spp, cur_spp, tmp);
    }
    return cudaGetLastError();
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
        k_weighted_sum_accumulate<__half><<<image_grid(g), dim3(32, 8), 0, s>>>(
            g, frame, second_alpha, weights, mins_maxs, cur_n, cur_p, filtered, prev_pix, accept, albedo,
            tone_mapped, cur_spp, (const __half*)acc_prev, (__half*)acc_cur);
    else
        k_weighted_sum_accumulate<float><<<image_grid(g), dim3(32, 8), 0, s>>>(
            g, frame, second_alpha, weights, mins_maxs, cur_n, cur_p, filtered, prev_pix, accept, albedo,
            tone_mapped, cur_spp, (const float*)acc_prev, (float*)acc_cur);
    return cudaGetLastError();
}

cudaError_t launch_taa(const Geometry& g, int frame, float taa_alpha, const float2* prev_pix,
                       const float* new_frame, void* result, const void* prev_frame, float* result_f32,
                       bool half_history, cudaStream_t s) {
    if (half_history)
        k_taa<__half><<<image_grid(g), dim3(32, 8), 0, s>>>(g, frame, taa_alpha, prev_pix, new_frame,
                                                           (__half*)result, (const __half*)prev_frame,
                                                           result_f32);
    else
        k_taa<float><<<image_grid(g), dim3(32, 8), 0, s>>>(g, frame, taa_alpha, prev_pix, new_frame,
                                                          (float*)result, (const float*)prev_frame,
                                                          result_f32);
    return cudaGetLastError();
}

}  // namespace bmfr
