// pixel_ops.cuh — per-pixel bodies of the BMFR stages (opencl/bmfr.cl),
// shared by the stage kernels and the fused per-block kernel.  Every float
// expression keeps the reference's operation order.
#pragma once

#include "common.cuh"

namespace bmfr {

__device__ __forceinline__ float3 hist_load(const float* p, int i) { return load3(p, i); }
__device__ __forceinline__ float3 hist_load(const __half* p, int i) {
    return make_float3(__half2float(p[3 * i]), __half2float(p[3 * i + 1]), __half2float(p[3 * i + 2]));
}

struct AccumResult {
    float ppx, ppy;      // prev_frame_pixel_f
    float3 color;        // blended colour
    uint8_t accept;
    uint8_t spp;
};

// Reprojection, 4-tap history gather and blend of one pixel
// (bmfr.cl:319-445).  `cur` is the pixel's colour before blending.
template <typename HistT>
__device__ __forceinline__ AccumResult accumulate_core(
    const Geometry& g, const AccumArgs& a, int px, int py, float3 wp, float3 nrm, float3 cur,
    const float* __restrict__ prev_n, const float* __restrict__ prev_p,
    const HistT* __restrict__ prev_noisy, const uint8_t* __restrict__ prev_spp) {
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
                        const float3 pc = hist_load(prev_noisy, s);
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

// weighted_sum body (bmfr.cl:712-750).
// Index of the block whose weights pixel (px, py) uses (bmfr.cl:718-722).
__device__ __forceinline__ int pixel_block(const Geometry& g, int frame, int px, int py) {
    const int2 bo = c_block_offsets[frame & 15];
    const int opx = px + kBlockEdge / 2 - bo.x, opy = py + kBlockEdge / 2 - bo.y;
    return (opx / kBlockEdge) + (opy / kBlockEdge) * g.MWb;
}

// w: the block's 30 weights, mm: its 12 min/max values.
__device__ __forceinline__ float3 weighted_sum_px(float3 wp, float3 n, const float* w, const float* mm) {
    const float f[kFeatures] = {1.0f, n.x, n.y, n.z, wp.x, wp.y, wp.z, wp.x * wp.x, wp.y * wp.y, wp.z * wp.z};
    float3 c = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < kFeatures; ++k) {
        float v = f[k];
        if (k >= kNotScaled) v = scale(v, mm[(k - kNotScaled) * 2], mm[(k - kNotScaled) * 2 + 1]);
        c.x = c.x + w[3 * k] * v;
        c.y = c.y + w[3 * k + 1] * v;
        c.z = c.z + w[3 * k + 2] * v;
    }
    c.x = c.x < 0.f ? 0.f : c.x;
    c.y = c.y < 0.f ? 0.f : c.y;
    c.z = c.z < 0.f ? 0.f : c.z;
    return c;
}

// accumulate_filtered_data body (bmfr.cl:778-856); returns the accumulated
// colour and writes the tone-mapped one through `tm`.
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

}  // namespace bmfr
