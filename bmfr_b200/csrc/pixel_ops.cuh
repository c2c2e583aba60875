// pixel_ops.cuh — per-pixel bodies of the BMFR stages (opencl/bmfr.cl),
// shared by the stage kernels and the fused per-block kernel.  Every float
// expression keeps the reference's operation order.
#pragma once

#include <type_traits>

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
// PREFETCH: the previous positions and normals of all in-image taps are
// loaded before any tap is tested, so their latencies overlap (more
// registers); the tests and the blend keep the reference's order either
// way.  Measured on the float-history pipeline at 1280x720: 159.1 -> 156.2 us
// per frame, and 184.7 -> 170.2 us in the fused block kernel; with binary16
// histories it lost (1080p 218.4 -> 220.4 us), so it is off there.
template <typename HistT, bool PREFETCH = std::is_same<HistT, float>::value>
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
        float3 tp[4], tn[4];
        int ts[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int sx = ix + (i & 1), sy = iy + (i >> 1);
            ts[i] = (sx >= 0 && sy >= 0 && sx < g.W && sy < g.H) ? sy * g.W + sx : -1;
            if (PREFETCH && ts[i] >= 0) {
                tp[i] = load3(prev_p, ts[i]);
                tn[i] = load3(prev_n, ts[i]);
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (ts[i] >= 0) {
                const int s = ts[i];
                const float3 pp = PREFETCH ? tp[i] : load3(prev_p, s);
                const float dx = pp.x - wp.x, dy = pp.y - wp.y, dz = pp.z - wp.z;
                if ((dx * dx + dy * dy) + dz * dz < a.pos_lim2) {
                    const float3 pn = PREFETCH ? tn[i] : load3(prev_n, s);
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

// accumulate_noisy_data of margin pixel (gx, gy) (bmfr.cl:310-484), out of
// place: the pixel's colour is read from noisy_in and the blended colour
// goes to the history noisy_out; in-image pixels also write spp,
// prev_frame_pixel and accept.
template <typename HistT>
__device__ __forceinline__ void accumulate_margin_px(
    const Geometry& g, const AccumArgs& a, int gx, int gy, float2* __restrict__ prev_pix,
    uint8_t* __restrict__ accept, const float* __restrict__ cur_n, const float* __restrict__ prev_n,
    const float* __restrict__ cur_p, const float* __restrict__ prev_p, const float* __restrict__ noisy_in,
    HistT* __restrict__ noisy_out, const HistT* __restrict__ prev_noisy, const uint8_t* __restrict__ prev_spp,
    uint8_t* __restrict__ cur_spp, void* __restrict__ tmp) {
    const int2 bo = c_block_offsets[a.frame & 15];
    const int pwx = gx - kBlockEdge / 2 + bo.x;
    const int pwy = gy - kBlockEdge / 2 + bo.y;
    const bool in_image = pwx >= 0 && pwx < g.W && pwy >= 0 && pwy < g.H;
    const int px = mirror(pwx, g.W), py = mirror(pwy, g.H);
    const int lp = py * g.W + px;
    const float3 wp = load3(cur_p, lp);
    const float3 nrm = load3(cur_n, lp);
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
// powr is evaluated as exp2(0.454545 * log2(x)) on the special function
// unit (__log2f, exp2f): relative error below 1e-6 for x above 1e-3 and a
// negligible absolute error below that (the OpenCL powr it stands for may
// be 16 ulp off); several times cheaper than powf.
__device__ __forceinline__ float tonemap1(float albedo, float acc) {
    const float x = fmax_cl(0.0f, albedo * acc);
    const float t = x > 0.0f ? exp2f(0.454545f * __log2f(x)) : 0.0f;
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

// weighted_sum followed by accumulate_filtered_data for image pixel (px, py)
// (bmfr.cl:712-757, 773-856), without stores: returns the accumulated
// colour, and the filtered and tone-mapped colours through `filt`, `tm`.
template <typename HistT>
__device__ __forceinline__ float3 wsacc_core(const Geometry& g, int frame, float second_alpha, int px, int py,
                                             const float* __restrict__ weights,
                                             const float* __restrict__ mins_maxs, const float* __restrict__ cur_n,
                                             const float* __restrict__ cur_p, const float2* __restrict__ prev_pix,
                                             const uint8_t* __restrict__ accept, const float* __restrict__ albedo,
                                             const uint8_t* __restrict__ cur_spp,
                                             const HistT* __restrict__ acc_prev, float3* filt, float3* tm) {
    const int lp = py * g.W + px;
    const int gi = pixel_block(g, frame, px, py);
    const float3 f = weighted_sum_px(load3(cur_p, lp), load3(cur_n, lp), weights + (size_t)gi * kFeatures * 3,
                                     mins_maxs + (size_t)gi * kScaled * 2);
    *filt = f;
    // The accumulation writes the reprojected position and spp of every
    // image pixel, so they are read beside the accept mask instead of after
    // it: the history gather then waits for one round trip, not two.  With
    // no accepted tap they go unused.
    const uint8_t acc = frame > 0 ? accept[lp] : 0;
    const float2 pp = frame > 0 ? prev_pix[lp] : make_float2(0.f, 0.f);
    const uint8_t spp = frame > 0 ? cur_spp[lp] : 1;
    return accumulate_filtered_px(g, frame, lp, f, pp, acc, spp, second_alpha, acc_prev, load3(albedo, lp), tm);
}

// wsacc_core with the stores of the separate stages; `filtered` may be null.
template <typename HistT>
__device__ __forceinline__ void wsacc_px(const Geometry& g, int frame, float second_alpha, int px, int py,
                                         const float* __restrict__ weights, const float* __restrict__ mins_maxs,
                                         const float* __restrict__ cur_n, const float* __restrict__ cur_p,
                                         float* __restrict__ filtered, const float2* __restrict__ prev_pix,
                                         const uint8_t* __restrict__ accept, const float* __restrict__ albedo,
                                         float* __restrict__ tone_mapped, const uint8_t* __restrict__ cur_spp,
                                         const HistT* __restrict__ acc_prev, HistT* __restrict__ acc_cur) {
    const int lp = py * g.W + px;
    float3 f, tm;
    const float3 a3 = wsacc_core<HistT>(g, frame, second_alpha, px, py, weights, mins_maxs, cur_n, cur_p, prev_pix,
                                        accept, albedo, cur_spp, acc_prev, &f, &tm);
    if (filtered) store3(filtered, lp, f);
    hist_store(acc_cur, lp, a3);
    store3(tone_mapped, lp, tm);
}

// taa body (bmfr.cl:873-973).
// YCoCg of one colour, unnormalised (bmfr.cl:184-198).
__device__ __forceinline__ void rgb_to_ycocg(float3 s, float (&ycc)[3]) {
    ycc[0] = (s.x * 1.0f + s.y * 2.0f) + s.z * 1.0f;
    ycc[1] = (s.x * 2.0f + s.y * 0.0f) + s.z * -2.0f;
    ycc[2] = (s.x * -1.0f + s.y * 2.0f) + s.z * -1.0f;
}

// The second half of taa (bmfr.cl:904-973) for pixel (px, py) whose
// tonemapped colour is `mine`, given the YCoCg bounds of its 3x3 box and
// its cross: history bilinear, clamp, blend.
template <typename HistT>
__device__ __forceinline__ float3 taa_finish(const Geometry& g, float taa_alpha, float2 pp, int ix, int iy,
                                             float3 mine, const float (&mnb)[3], const float (&mxb)[3],
                                             const float (&mnc)[3], const float (&mxc)[3],
                                             const HistT* __restrict__ prev_frame) {
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
    float pyc[3];
    rgb_to_ycocg(prev, pyc);
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

// taa (bmfr.cl:868-973) of pixel (px, py) whose tonemapped colour is `mine`;
// nb(x, y, ycc) gives the YCoCg of the in-image neighbour (px+x, py+y).
template <typename HistT, typename Nb>
__device__ __forceinline__ float3 taa_core(const Geometry& g, int frame, float taa_alpha, int px, int py, float2 pp,
                                           float3 mine, Nb&& nb, const HistT* __restrict__ prev_frame) {
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
                float ycc[3];
                nb(x, y, ycc);
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
    return taa_finish(g, taa_alpha, pp, ix, iy, mine, mnb, mxb, mnc, mxc, prev_frame);
}

// taa over a strip of R rows per thread.  A warp covers 30 image columns
// x0..x0+29 in lanes 1..30 (lanes 0 and 31 hold the halo columns) and walks
// rows y0..y0+R-1: each thread reads and converts one pixel per row (R+2
// rows with the halo), takes its left and right neighbours by shuffles, and
// keeps a three-row window of horizontal minima and maxima, so a pixel's
// nine neighbours cost about one load and one YCoCg conversion.  Neighbours
// outside the image or NaN enter as +-inf, which the reference's fmin/fmax
// ignore in the same way (bmfr.cl:884-902; fmin/fmax return the other
// operand of a NaN), so the bounds equal the reference's up to the sign of a
// zero bound.
template <int R, typename HistT>
__device__ __forceinline__ void taa_strip(const Geometry& g, int frame, float taa_alpha, int x0, int y0,
                                          const float2* __restrict__ prev_pix, const float* __restrict__ new_frame,
                                          const HistT* __restrict__ prev_frame, HistT* __restrict__ result_hist,
                                          float* __restrict__ result_out) {
    const int lane = threadIdx.x & 31;
    const int x = x0 - 1 + lane;
    const bool col_in = x >= 0 && x < g.W;
    const bool writer = lane >= 1 && lane <= 30 && col_in;
    float3 rgb[3];
    float cmn[3][3], cmx[3][3], hmn[3][3], hmx[3][3];   // [window row][channel]
    // The strip's reprojected positions first: the history gather of each
    // row depends on them, and they depend on nothing here (1920x1080
    // frame 319.4 -> 315.2 us).
    float2 ppre[R];
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
        const int py = y0 + rr;
        ppre[rr] = (writer && py < g.H) ? prev_pix[py * g.W + x] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int r = 0; r < R + 2; ++r) {
        const int k = r % 3;
        const int y = y0 - 1 + r;
        const bool in = col_in && y >= 0 && y < g.H;
        const float3 s = in ? load3(new_frame, y * g.W + x) : make_float3(0.f, 0.f, 0.f);
        rgb[k] = s;
        float ycc[3];
        rgb_to_ycocg(s, ycc);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            // Out-of-image entries as NaN, which fminf/fmaxf skip (they
            // return the other operand), so one shuffle each way serves both
            // bounds; the pixel's own candidates turn a NaN into +-inf.
            // Lanes 0 and 31, the halo columns, take their own as a
            // neighbour and are not written.
            const float v = in ? ycc[c] : __int_as_float(0x7fffffff);
            const float vl = __shfl_up_sync(0xffffffffu, v, 1), vr = __shfl_down_sync(0xffffffffu, v, 1);
            const float vmn = fminf(v, INFINITY), vmx = fmaxf(v, -INFINITY);
            cmn[k][c] = vmn;
            cmx[k][c] = vmx;
            hmn[k][c] = fminf(fminf(vl, vmn), vr);
            hmx[k][c] = fmaxf(fmaxf(vl, vmx), vr);
        }
        if (r >= 2) {
            const int up = (r - 2) % 3, mid = (r - 1) % 3, dn = k;
            const int py = y0 + r - 2;
            if (writer && py < g.H) {
                const int lp = py * g.W + x;
                const float2 pp = ppre[r - 2];
                const float3 mine = rgb[mid];
                const int ix = floor_to_int(pp.x), iy = floor_to_int(pp.y);
                float3 out = mine;
                if (!(frame == 0 || ix < -1 || iy < -1 || ix >= g.W || iy >= g.H)) {
                    float mnb[3], mxb[3], mnc[3], mxc[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        mnb[c] = fminf(fminf(hmn[up][c], hmn[mid][c]), hmn[dn][c]);
                        mxb[c] = fmaxf(fmaxf(hmx[up][c], hmx[mid][c]), hmx[dn][c]);
                        mnc[c] = fminf(fminf(cmn[up][c], hmn[mid][c]), cmn[dn][c]);
                        mxc[c] = fmaxf(fmaxf(cmx[up][c], hmx[mid][c]), cmx[dn][c]);
                    }
                    out = taa_finish(g, taa_alpha, pp, ix, iy, mine, mnb, mxb, mnc, mxc, prev_frame);
                }
                hist_store(result_hist, lp, out);
                if (result_out) store3(result_out, lp, out);
            }
        }
    }
}

// taa of one pixel, neighbours read from global memory.
template <typename HistT>
__device__ __forceinline__ float3 taa_px(const Geometry& g, int frame, float taa_alpha, int px, int py,
                                         float2 pp, const float* __restrict__ new_frame,
                                         const HistT* __restrict__ prev_frame) {
    const float3 mine = load3(new_frame, py * g.W + px);
    auto nb = [&](int x, int y, float (&ycc)[3]) {
        const float3 s = (x == 0 && y == 0) ? mine : load3(new_frame, (py + y) * g.W + px + x);
        rgb_to_ycocg(s, ycc);
    };
    return taa_core(g, frame, taa_alpha, px, py, pp, mine, nb, prev_frame);
}


}  // namespace bmfr
