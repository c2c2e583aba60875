// bmfr_oracle.cpp — TEST INFRASTRUCTURE ONLY: CPU restatement of the
// reference's OpenCL kernels (opencl/bmfr.cl), the parity checker of the CUDA
// pipeline and the timed CPU baseline.  Nothing in the product links this.
//
// PINNED to the reference itself: the reference's own kernels, compiled for
// the CPU by oracle/ref_cl, give bit-identical outputs on the same inputs
// (tests/test_reference_pin.py, fixtures in tests/golden/).
//
// Arithmetic rules (compiled with -ffp-contract=off, no fast-math):
//  * every float expression keeps the reference's evaluation order, one
//    rounding per operation, no fused multiply-add;
//  * dot(a, b) of OpenCL vectors is evaluated left to right,
//    ((a.x*b.x + a.y*b.y) + a.z*b.z) + a.w*b.w;
//  * vstore_half rounds to nearest even (bmfr.cl:255-258);
//  * convert_int2_rtn is floor; NaN and values beyond +-2^30 map to -2^30 /
//    +2^30 so that they land outside every image (OpenCL leaves the
//    conversion of out-of-range values undefined);
//  * fmin/fmax are (y < x ? y : x) / (x < y ? y : x), returning the other
//    operand when x is NaN (the specification's NaN rule; max(0, v) of the
//    tone map gives the same values);
//  * the fitter's work-group reductions are evaluated over the same tree as
//    parallel_reduction_sum/min/max (bmfr.cl:25-87).
#include "bmfr_oracle.h"

#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int kBlock = 32;           // BLOCK_EDGE_LENGTH
constexpr int kBlockPixels = 1024;   // BLOCK_PIXELS
constexpr int kLocal = 256;          // LOCAL_SIZE
constexpr int kBuffers = 13;         // BUFFER_COUNT
constexpr int kNotScaled = 4;        // FEATURES_NOT_SCALED
constexpr int kScaled = 6;           // FEATURES_SCALED
constexpr int kREdge = 11;           // R_EDGE

// bmfr.cl:268-285
const int kBlockOffsets[16][2] = {
    {-14, -14}, {4, -6}, {-8, 14}, {8, 0}, {-10, -8}, {2, 12}, {12, -12},
    {-10, 0}, {12, 14}, {-8, -16}, {6, 6}, {-2, -2}, {6, -14}, {-16, 12},
    {14, -4}, {-6, 4}};

inline float half_round(float v) { return (float)(_Float16)v; }

// OpenCL fmin/fmax: y if y < x (x < y), else x; the other operand when x is
// NaN (a NaN reaches the clamp of taa when all history weights are zero).
inline float fmin_cl(float x, float y) { return (y < x || x != x) ? y : x; }
inline float fmax_cl(float x, float y) { return (x < y || x != x) ? y : x; }

// convert_int_rtn with defined results outside the int range.
inline int floor_to_int(float v) {
    if (!(v == v)) return -(1 << 30);
    float f = std::floor(v);
    if (f < -1073741824.0f) return -(1 << 30);
    if (f > 1073741824.0f) return 1 << 30;
    return (int)f;
}

// bmfr.cl:209-216
inline int mirror(int index, int size) {
    if (index < 0)
        index = std::abs(index) - 1;
    else if (index >= size)
        index = 2 * size - index - 1;
    return index;
}

// bmfr.cl:162-171 (hash from asgerhoedt.dk/?p=323).
inline float random_u32(uint32_t a) {
    a = (a + 0x7ed55d16u) + (a << 12);
    a = (a ^ 0xc761c23cu) ^ (a >> 19);
    a = (a + 0x165667b1u) + (a << 5);
    a = (a + 0xd3a2646cu) ^ (a << 9);
    a = (a + 0xfd7046c5u) + (a << 3);
    a = (a ^ 0xb55a4f09u) ^ (a >> 16);
    // convert_float(a) / convert_float(UINT_MAX): both round to nearest.
    return (float)a / (float)4294967295u;
}

inline uint32_t noise_index(int id, int sub_vector, int feature_buffer, int frame) {
    // bmfr.cl:179-181, int arithmetic wrapped to unsigned.
    return (uint32_t)id + (uint32_t)sub_vector * (uint32_t)kLocal +
           (uint32_t)feature_buffer * (uint32_t)kBlockPixels +
           (uint32_t)frame * (uint32_t)(kBuffers * kBlockPixels);
}

// bmfr.cl:173-182.  NOISE_AMOUNT is the double literal 1e-2, so
// NOISE_AMOUNT * 2.f * (r - 0.5f) and the sum are formed in double and the
// result is rounded once to float on return.
inline float add_random(float value, int id, int sv, int fb, int frame, double noise) {
    float r = random_u32(noise_index(id, sv, fb, frame)) - 0.5f;
    double v = (double)value + (noise * 2.0) * (double)r;
    return (float)v;
}
inline double add_random_d(double value, int id, int sv, int fb, int frame, double noise) {
    float r = random_u32(noise_index(id, sv, fb, frame)) - 0.5f;
    return value + (noise * 2.0) * (double)r;
}

inline float scale(float value, float mn, float mx) {   // bmfr.cl:200-205
    if (std::fabs(mx - mn) > 1.0f) return (value - mn) / (mx - mn);
    return value - mn;
}
inline double scale_d(double value, double mn, double mx) {
    if (std::fabs(mx - mn) > 1.0) return (value - mn) / (mx - mn);
    return value - mn;
}

inline float dot3(const float* a, const float* b) {
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}

// parallel_reduction_sum (bmfr.cl:26-44) over 256 work-item values.
template <typename T>
T reduce_sum(T* sv) {
    for (int id = 0; id < 64; ++id)
        sv[id] = sv[id] + ((sv[id + 64] + sv[id + 128]) + sv[id + 192]);
    for (int id = 0; id < 8; ++id)
        sv[id] = sv[id] + ((((((sv[id + 8] + sv[id + 16]) + sv[id + 24]) + sv[id + 32]) +
                             sv[id + 40]) + sv[id + 48]) + sv[id + 56]);
    return ((((((sv[0] + sv[1]) + sv[2]) + sv[3]) + sv[4]) + sv[5]) + sv[6]) + sv[7];
}
// parallel_reduction_min / max (bmfr.cl:46-87).
template <bool MAX>
float reduce_minmax(float* sv) {
    auto op = [](float a, float b) { return MAX ? fmax_cl(a, b) : fmin_cl(a, b); };
    for (int id = 0; id < 64; ++id)
        sv[id] = op(op(op(sv[id], sv[id + 64]), sv[id + 128]), sv[id + 192]);
    for (int id = 0; id < 8; ++id) {
        float v = sv[id];
        for (int m = 1; m < 8; ++m) v = op(v, sv[id + 8 * m]);
        sv[id] = v;
    }
    float r = sv[0];
    for (int m = 1; m < 8; ++m) r = op(r, sv[m]);
    return r;
}

int threads_of(const orc_cfg* c) {
#ifdef _OPENMP
    return c->threads > 0 ? c->threads : omp_get_max_threads();
#else
    (void)c;
    return 1;
#endif
}

struct Geometry {
    int W, H, WW, WH, MW, MH, MWb, MHb, B;
    explicit Geometry(const orc_cfg* c) {
        W = c->width;
        H = c->height;
        WW = kBlock * ((W + kBlock - 1) / kBlock);   // WORKSET_WIDTH (bmfr.cpp:107)
        WH = kBlock * ((H + kBlock - 1) / kBlock);
        MW = WW + kBlock;                            // WORKSET_WITH_MARGINS_WIDTH
        MH = WH + kBlock;
        MWb = MW / kBlock;
        MHb = MH / kBlock;
        B = MWb * MHb;                               // FITTER_GLOBAL / LOCAL_SIZE
    }
};

// Per-margin-pixel body of accumulate_noisy_data (bmfr.cl:310-476).  Writes the
// 13 tmp values and returns the owner-only outputs through the pointers.
struct AccumOut {
    float prev_pixel[2];
    uint8_t accept;
    uint8_t spp;
    float new_color[3];
    int linear_pixel;
    bool in_image;
};

AccumOut accumulate_pixel(const orc_cfg* cfg, const Geometry& g, int gx, int gy,
                          const float* cur_n, const float* prev_n, const float* cur_p,
                          const float* prev_p, const float* raw_noisy,
                          const float* prev_noisy, const uint8_t* prev_spp,
                          const float* M, const float* off, int frame, void* tmp) {
    AccumOut o;
    const int* bo = kBlockOffsets[frame % 16];
    const int pwx = gx - kBlock / 2 + bo[0];
    const int pwy = gy - kBlock / 2 + bo[1];
    const int px = mirror(pwx, g.W), py = mirror(pwy, g.H);
    const int lp = py * g.W + px;
    o.linear_pixel = lp;
    o.in_image = pwx >= 0 && pwx < g.W && pwy >= 0 && pwy < g.H;

    const float wp[4] = {cur_p[lp * 3], cur_p[lp * 3 + 1], cur_p[lp * 3 + 2], 1.0f};
    const float nrm[3] = {cur_n[lp * 3], cur_n[lp * 3 + 1], cur_n[lp * 3 + 2]};
    const float cc[3] = {raw_noisy[lp * 3], raw_noisy[lp * 3 + 1], raw_noisy[lp * 3 + 2]};

    float ppf[2] = {(float)px, (float)py};
    uint8_t accept = 0;
    float alpha = 1.0f;
    float prev[3] = {0.f, 0.f, 0.f};
    float sample_spp = 0.0f;
    if (frame > 0) {
        // s048c, s159d, s37bf (bmfr.cl:343-347)
        float uvx = ((M[0] * wp[0] + M[4] * wp[1]) + M[8] * wp[2]) + M[12] * wp[3];
        float uvy = ((M[1] * wp[0] + M[5] * wp[1]) + M[9] * wp[2]) + M[13] * wp[3];
        float w = ((M[3] * wp[0] + M[7] * wp[1]) + M[11] * wp[2]) + M[15] * wp[3];
        uvx = uvx / w;
        uvy = uvy / w;
        uvx = uvx + 1.0f;
        uvy = uvy + 1.0f;
        uvx = uvx / 2.0f;
        uvy = uvy / 2.0f;
        ppf[0] = uvx * (float)g.W;
        ppf[1] = uvy * (float)g.H;
        ppf[0] = ppf[0] - off[0];
        ppf[1] = ppf[1] - (1.0f - off[1]);
        const int ix = floor_to_int(ppf[0]), iy = floor_to_int(ppf[1]);
        const float fx = ppf[0] - (float)ix, fy = ppf[1] - (float)iy;
        const float ofx = 1.0f - fx, ofy = 1.0f - fy;
        const float wts[4] = {ofx * ofy, fx * ofy, ofx * fy, fx * fy};
        const int ox[4] = {0, 1, 0, 1}, oy[4] = {0, 0, 1, 1};
        float total = 0.0f;
        for (int i = 0; i < 4; ++i) {
            const int sx = ix + ox[i], sy = iy + oy[i];
            if (sx >= 0 && sy >= 0 && sx < g.W && sy < g.H) {
                const int s = sy * g.W + sx;
                const float pd[3] = {prev_p[s * 3] - wp[0], prev_p[s * 3 + 1] - wp[1],
                                     prev_p[s * 3 + 2] - wp[2]};
                if (dot3(pd, pd) < cfg->position_limit_squared) {
                    const float nd[3] = {prev_n[s * 3] - nrm[0], prev_n[s * 3 + 1] - nrm[1],
                                         prev_n[s * 3 + 2] - nrm[2]};
                    if (dot3(nd, nd) < cfg->normal_limit_squared) {
                        accept |= (uint8_t)(1 << i);
                        sample_spp = sample_spp + wts[i] * (float)prev_spp[s];
                        for (int c = 0; c < 3; ++c)
                            prev[c] = prev[c] + wts[i] * prev_noisy[s * 3 + c];
                        total = total + wts[i];
                    }
                }
            }
        }
        if (total > 0.0f) {
            for (int c = 0; c < 3; ++c) prev[c] = prev[c] / total;
            sample_spp = sample_spp / total;
            alpha = 1.0f / (sample_spp + 1.0f);
            alpha = fmax_cl(alpha, cfg->blend_alpha);
        }
    }
    uint8_t new_spp = 1;   // bmfr.cl:433-441
    if (alpha < 1.0f) {
        if (sample_spp > 254.0f) {
            new_spp = 255;
        } else {
            float r = std::nearbyint(sample_spp);   // round to nearest even
            r = r < 0.f ? 0.f : (r > 255.f ? 255.f : r);
            new_spp = (uint8_t)((int)r + 1);
        }
    }
    o.spp = new_spp;
    const float one_minus = 1.0f - alpha;
    for (int c = 0; c < 3; ++c) o.new_color[c] = alpha * cc[c] + one_minus * prev[c];

    const float feats[kBuffers] = {1.0f, nrm[0], nrm[1], nrm[2], wp[0], wp[1], wp[2],
                                   wp[0] * wp[0], wp[1] * wp[1], wp[2] * wp[2],
                                   o.new_color[0], o.new_color[1], o.new_color[2]};
    const int xin = gx % kBlock, yin = gy % kBlock, xb = gx / kBlock, yb = gy / kBlock;
    const size_t base = ((size_t)(yb * g.MWb + xb) * kBuffers) * kBlockPixels +
                        (size_t)(yin * kBlock + xin);
    for (int k = 0; k < kBuffers; ++k) {
        float v = feats[k];
        if (std::isnan(v)) v = 0.0f;
        if (cfg->use_half) {
            v = std::max(std::min(v, 65504.0f), -65504.0f);
            ((_Float16*)tmp)[base + (size_t)k * kBlockPixels] = (_Float16)v;
        } else {
            ((float*)tmp)[base + (size_t)k * kBlockPixels] = v;
        }
    }
    o.prev_pixel[0] = ppf[0];
    o.prev_pixel[1] = ppf[1];
    o.accept = accept;
    return o;
}

// The fitter over one block (bmfr.cl:503-699) in the reference's arithmetic.
// `tile` holds the block's 13 columns as floats; stq() is the STORE rounding.
void fit_block_fp32(float* tile, float* weights_out, float* mm_out, int frame,
                    double noise, bool round_half_stores) {
    auto stq = [&](float v) { return round_half_stores ? half_round(v) : v; };
    float sv[kLocal];

    // Scaling of the position features (bmfr.cl:511-542).
    for (int fb = kNotScaled; fb < kBuffers - 3; ++fb) {
        float* col = tile + fb * kBlockPixels;
        float tmax[kLocal], tmin[kLocal];
        for (int id = 0; id < kLocal; ++id) {
            float mx = -INFINITY, mn = INFINITY;
            for (int s = 0; s < 4; ++s) {
                const float v = col[id + s * kLocal];
                mx = fmax_cl(v, mx);
                mn = fmin_cl(v, mn);
            }
            tmax[id] = mx;
            tmin[id] = mn;
        }
        std::memcpy(sv, tmax, sizeof sv);
        const float bmax = reduce_minmax<true>(sv);
        std::memcpy(sv, tmin, sizeof sv);
        const float bmin = reduce_minmax<false>(sv);
        mm_out[(fb - kNotScaled) * 2 + 0] = bmin;
        mm_out[(fb - kNotScaled) * 2 + 1] = bmax;
        for (int i = 0; i < kBlockPixels; ++i) col[i] = stq(scale(col[i], bmin, bmax));
    }

    // Householder QR, column by column (bmfr.cl:546-656).  R is kept dense:
    // R[x][y][channel], x = column, y = row.  The compressed layout of the
    // reference (bmfr.cl:100-103) only changes where values live; the slots it
    // aliases are rewritten by later columns before they are read.
    float R[kREdge][kREdge][3];
    std::memset(R, 0, sizeof R);
    float u[kBlockPixels];
    for (int col = 0; col < kBuffers; ++col) {
        const int cl = std::min(col, kBuffers - 3);
        const float* a = tile + col * kBlockPixels;
        for (int id = 0; id < kLocal; ++id) {
            float s = 0.0f;
            for (int q = 0; q < 4; ++q) {
                const int idx = id + q * kLocal;
                u[idx] = a[idx];
                if (idx >= cl + 1) s = s + a[idx] * a[idx];
            }
            sv[id] = s;
        }
        const float norm2 = reduce_sum(sv);
        // Work-item `col` (bmfr.cl:580-588); the others copy u or zero.
        float uls = norm2;
        const float vl = std::sqrt(norm2 + u[cl] * u[cl]);
        const float u_cl_before = u[cl];
        u[cl] = u[cl] - vl;
        uls = uls + u[cl] * u[cl];
        if (col < kBuffers - 3) {
            for (int y = 0; y <= kREdge - 1; ++y) {
                const float r = y < col ? u[y] : (y == col ? vl : 0.0f);
                for (int c = 0; c < 3; ++c) R[col][y][c] = r;
            }
        } else {
            const int ch = col - (kBuffers - 3);
            for (int y = 0; y < kREdge - 1; ++y) R[kREdge - 1][y][ch] = u[y];
            (void)u_cl_before;   // R[10][10] is never read (bmfr.cl:660-699)
        }
        // Transform the later columns (bmfr.cl:606-655).
        for (int fb = cl + 1; fb < kBuffers; ++fb) {
            float* t = tile + fb * kBlockPixels;
            float cache[kBlockPixels];
            for (int id = 0; id < kLocal; ++id) {
                float s = 0.0f;
                for (int q = 0; q < 4; ++q) {
                    const int idx = id + q * kLocal;
                    if (idx >= cl) {
                        float v = t[idx];
                        if (col == 0 && fb < kBuffers - 3)
                            v = add_random(v, id, q, fb, frame, noise);
                        cache[idx] = v;
                        s = s + v * u[idx];
                    }
                }
                sv[id] = s;
            }
            const float dot = reduce_sum(sv);
            for (int idx = cl; idx < kBlockPixels; ++idx)
                t[idx] = stq(cache[idx] - ((2.0f * u[idx]) * dot) / uls);
        }
    }

    // Back substitution (bmfr.cl:659-692).
    for (int i = kREdge - 2; i >= 0; --i) {
        float d[3] = {R[i][i][0], R[i][i][1], R[i][i][2]};
        for (int x = i; x < kREdge; ++x)
            for (int c = 0; c < 3; ++c) R[x][i][c] = R[x][i][c] / d[c];
        for (int j = i + 1; j < kREdge - 1; ++j)
            for (int c = 0; c < 3; ++c) R[kREdge - 1][i][c] = R[kREdge - 1][i][c] - R[j][i][c];
        for (int y = 0; y <= i; ++y)
            for (int c = 0; c < 3; ++c) R[i][y][c] = R[i][y][c] * R[kREdge - 1][i][c];
    }
    for (int k = 0; k < kBuffers - 3; ++k)
        for (int c = 0; c < 3; ++c) weights_out[k * 3 + c] = R[kREdge - 1][k][c];
}

// fp64 restatement: the same steps and reduction trees in double precision,
// with no intermediate rounding of the block.
void fit_block_fp64(const float* tile_in, double* weights_out, float* mm_out, int frame,
                    double noise) {
    std::vector<double> tile(kBuffers * kBlockPixels);
    for (int i = 0; i < kBuffers * kBlockPixels; ++i) tile[i] = tile_in[i];
    double sv[kLocal];
    for (int fb = kNotScaled; fb < kBuffers - 3; ++fb) {
        double* col = tile.data() + fb * kBlockPixels;
        float bmax = -INFINITY, bmin = INFINITY;   // min/max are exact
        for (int i = 0; i < kBlockPixels; ++i) {
            bmax = fmax_cl((float)col[i], bmax);
            bmin = fmin_cl((float)col[i], bmin);
        }
        mm_out[(fb - kNotScaled) * 2 + 0] = bmin;
        mm_out[(fb - kNotScaled) * 2 + 1] = bmax;
        for (int i = 0; i < kBlockPixels; ++i) col[i] = scale_d(col[i], bmin, bmax);
    }
    double R[kREdge][kREdge][3];
    std::memset(R, 0, sizeof R);
    std::vector<double> u(kBlockPixels), cache(kBlockPixels);
    // Columns 10..12 only reflect rows >= 10, which no output reads.
    for (int col = 0; col < kBuffers - 3; ++col) {
        const int cl = col;
        const double* a = tile.data() + col * kBlockPixels;
        for (int id = 0; id < kLocal; ++id) {
            double s = 0.0;
            for (int q = 0; q < 4; ++q) {
                const int idx = id + q * kLocal;
                u[idx] = a[idx];
                if (idx >= cl + 1) s = s + a[idx] * a[idx];
            }
            sv[id] = s;
        }
        const double norm2 = reduce_sum(sv);
        double uls = norm2;
        const double vl = std::sqrt(norm2 + u[cl] * u[cl]);
        u[cl] = u[cl] - vl;
        uls = uls + u[cl] * u[cl];
        for (int y = 0; y <= kREdge - 1; ++y) {
            const double r = y < col ? u[y] : (y == col ? vl : 0.0);
            for (int c = 0; c < 3; ++c) R[col][y][c] = r;
        }
        for (int fb = cl + 1; fb < kBuffers; ++fb) {
            double* t = tile.data() + fb * kBlockPixels;
            for (int id = 0; id < kLocal; ++id) {
                double s = 0.0;
                for (int q = 0; q < 4; ++q) {
                    const int idx = id + q * kLocal;
                    if (idx >= cl) {
                        double v = t[idx];
                        if (col == 0 && fb < kBuffers - 3)
                            v = add_random_d(v, id, q, fb, frame, noise);
                        cache[idx] = v;
                        s = s + v * u[idx];
                    }
                }
                sv[id] = s;
            }
            const double dot = reduce_sum(sv);
            for (int idx = cl; idx < kBlockPixels; ++idx)
                t[idx] = cache[idx] - ((2.0 * u[idx]) * dot) / uls;
        }
    }
    // RHS rows 0..9 of the colour columns after the ten reflections.
    for (int c = 0; c < 3; ++c)
        for (int y = 0; y < kREdge - 1; ++y)
            R[kREdge - 1][y][c] = tile[(kBuffers - 3 + c) * kBlockPixels + y];
    for (int i = kREdge - 2; i >= 0; --i) {
        double d[3] = {R[i][i][0], R[i][i][1], R[i][i][2]};
        for (int x = i; x < kREdge; ++x)
            for (int c = 0; c < 3; ++c) R[x][i][c] = R[x][i][c] / d[c];
        for (int j = i + 1; j < kREdge - 1; ++j)
            for (int c = 0; c < 3; ++c) R[kREdge - 1][i][c] = R[kREdge - 1][i][c] - R[j][i][c];
        for (int y = 0; y <= i; ++y)
            for (int c = 0; c < 3; ++c) R[i][y][c] = R[i][y][c] * R[kREdge - 1][i][c];
    }
    for (int k = 0; k < kBuffers - 3; ++k)
        for (int c = 0; c < 3; ++c) weights_out[k * 3 + c] = R[kREdge - 1][k][c];
}

void load_block(const orc_cfg* cfg, const void* tmp, int b, float* tile) {
    const size_t base = (size_t)b * kBuffers * kBlockPixels;
    for (int i = 0; i < kBuffers * kBlockPixels; ++i)
        tile[i] = cfg->use_half ? (float)((const _Float16*)tmp)[base + i]
                                : ((const float*)tmp)[base + i];
}
void store_block(const orc_cfg* cfg, void* tmp, int b, const float* tile) {
    const size_t base = (size_t)b * kBuffers * kBlockPixels;
    for (int i = 0; i < kBuffers * kBlockPixels; ++i) {
        if (cfg->use_half)
            ((_Float16*)tmp)[base + i] = (_Float16)tile[i];
        else
            ((float*)tmp)[base + i] = tile[i];
    }
}

}  // namespace

extern "C" {

void orc_sizes(const orc_cfg* cfg, int* margin_w, int* margin_h, int* blocks) {
    Geometry g(cfg);
    if (margin_w) *margin_w = g.MW;
    if (margin_h) *margin_h = g.MH;
    if (blocks) *blocks = g.B;
}

float orc_random(uint32_t a) { return random_u32(a); }
int orc_mirror(int index, int size) { return mirror(index, size); }
float orc_round_half(float v) { return half_round(v); }
float orc_add_random(float value, int id, int sub_vector, int feature_buffer,
                     int frame_number, double noise_amount) {
    return add_random(value, id, sub_vector, feature_buffer, frame_number, noise_amount);
}

void orc_accumulate_noisy_data(const orc_cfg* cfg, float* out_prev_frame_pixel,
                               uint8_t* accept_bools, const float* current_normals,
                               const float* previous_normals,
                               const float* current_positions,
                               const float* previous_positions, float* current_noisy,
                               const float* previous_noisy, const uint8_t* previous_spp,
                               uint8_t* current_spp, void* tmp_data,
                               const float* camera_matrix, const float* pixel_offset,
                               int frame_number) {
    Geometry g(cfg);
    // Every margin work-item reads the colour as it was before the kernel.
    std::vector<float> raw(current_noisy, current_noisy + (size_t)g.W * g.H * 3);
    const int nt = threads_of(cfg);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int gy = 0; gy < g.MH; ++gy) {
        for (int gx = 0; gx < g.MW; ++gx) {
            AccumOut o = accumulate_pixel(cfg, g, gx, gy, current_normals, previous_normals,
                                          current_positions, previous_positions, raw.data(),
                                          previous_noisy, previous_spp, camera_matrix,
                                          pixel_offset, frame_number, tmp_data);
            if (o.in_image) {   // bmfr.cl:478-484 (spp: every work-item, same value)
                current_spp[o.linear_pixel] = o.spp;
                for (int c = 0; c < 3; ++c) current_noisy[o.linear_pixel * 3 + c] = o.new_color[c];
                out_prev_frame_pixel[o.linear_pixel * 2 + 0] = o.prev_pixel[0];
                out_prev_frame_pixel[o.linear_pixel * 2 + 1] = o.prev_pixel[1];
                accept_bools[o.linear_pixel] = o.accept;
            }
        }
    }
}

void orc_fitter(const orc_cfg* cfg, float* weights, float* mins_maxs, void* tmp_data,
                int frame_number, int mode) {
    Geometry g(cfg);
    const int nt = threads_of(cfg);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int b = 0; b < g.B; ++b) {
        std::vector<float> tile(kBuffers * kBlockPixels);
        load_block(cfg, tmp_data, b, tile.data());
        if (mode == ORC_FITTER_FP64) {
            double w[30];
            fit_block_fp64(tile.data(), w, mins_maxs + b * kScaled * 2, frame_number,
                           cfg->noise_amount);
            for (int i = 0; i < 30; ++i) weights[b * 30 + i] = (float)w[i];
        } else {
            fit_block_fp32(tile.data(), weights + b * 30, mins_maxs + b * kScaled * 2,
                           frame_number, cfg->noise_amount,
                           mode == ORC_FITTER_REFERENCE && cfg->use_half);
            store_block(cfg, tmp_data, b, tile.data());
        }
    }
}

void orc_fitter_matrix(const orc_cfg* cfg, const void* tmp_data, int frame_number, double* out) {
    Geometry g(cfg);
    const int nt = threads_of(cfg);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int b = 0; b < g.B; ++b) {
        std::vector<float> tile(kBuffers * kBlockPixels);
        load_block(cfg, tmp_data, b, tile.data());
        double* m = out + (size_t)b * kBuffers * kBlockPixels;
        for (int i = 0; i < kBuffers * kBlockPixels; ++i) m[i] = tile[i];
        for (int fb = kNotScaled; fb < kBuffers - 3; ++fb) {
            double* col = m + fb * kBlockPixels;
            float bmax = -INFINITY, bmin = INFINITY;
            for (int i = 0; i < kBlockPixels; ++i) {
                bmax = fmax_cl((float)col[i], bmax);
                bmin = fmin_cl((float)col[i], bmin);
            }
            for (int i = 0; i < kBlockPixels; ++i) col[i] = scale_d(col[i], bmin, bmax);
        }
        for (int fb = 1; fb < kBuffers - 3; ++fb)
            for (int id = 0; id < kLocal; ++id)
                for (int q = 0; q < 4; ++q) {
                    const int idx = id + q * kLocal;
                    m[fb * kBlockPixels + idx] =
                        add_random_d(m[fb * kBlockPixels + idx], id, q, fb, frame_number, cfg->noise_amount);
                }
    }
}

void orc_fitter_fp64(const orc_cfg* cfg, double* weights, float* mins_maxs,
                     const void* tmp_data, int frame_number) {
    Geometry g(cfg);
    const int nt = threads_of(cfg);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int b = 0; b < g.B; ++b) {
        std::vector<float> tile(kBuffers * kBlockPixels);
        load_block(cfg, tmp_data, b, tile.data());
        fit_block_fp64(tile.data(), weights + b * 30, mins_maxs + b * kScaled * 2,
                       frame_number, cfg->noise_amount);
    }
}

void orc_weighted_sum(const orc_cfg* cfg, const float* weights, const float* mins_maxs,
                      float* output, const float* current_normals,
                      const float* current_positions, int frame_number) {
    Geometry g(cfg);
    const int* bo = kBlockOffsets[frame_number % 16];
    const int nt = threads_of(cfg);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int py = 0; py < g.H; ++py) {
        for (int px = 0; px < g.W; ++px) {
            const int lp = py * g.W + px;
            const int opx = px + kBlock / 2 - bo[0], opy = py + kBlock / 2 - bo[1];
            const int gi = (opx / kBlock) + (opy / kBlock) * g.MWb;
            const float* p = current_positions + lp * 3;
            const float* n = current_normals + lp * 3;
            const float f[10] = {1.0f, n[0], n[1], n[2], p[0], p[1], p[2],
                                 p[0] * p[0], p[1] * p[1], p[2] * p[2]};
            float color[3] = {0.f, 0.f, 0.f};
            for (int k = 0; k < 10; ++k) {
                float feat = f[k];
                if (k >= kNotScaled) {
                    const int mi = (gi * kScaled + k - kNotScaled) * 2;
                    feat = scale(feat, mins_maxs[mi], mins_maxs[mi + 1]);
                }
                const float* w = weights + (gi * 10 + k) * 3;
                for (int c = 0; c < 3; ++c) color[c] = color[c] + w[c] * feat;
            }
            for (int c = 0; c < 3; ++c) output[lp * 3 + c] = color[c] < 0.f ? 0.f : color[c];
        }
    }
}

void orc_accumulate_filtered_data(const orc_cfg* cfg, const float* filtered_frame,
                                  const float* in_prev_frame_pixel,
                                  const uint8_t* accept_bools, const float* albedo,
                                  float* tone_mapped_frame, const uint8_t* current_spp,
                                  const float* accumulated_prev_frame,
                                  float* accumulated_frame, int frame_number) {
    Geometry g(cfg);
    const int nt = threads_of(cfg);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int py = 0; py < g.H; ++py) {
        for (int px = 0; px < g.W; ++px) {
            const int lp = py * g.W + px;
            const float* fc = filtered_frame + lp * 3;
            float prev[3] = {0.f, 0.f, 0.f};
            float alpha = 1.0f;
            if (frame_number > 0) {
                const uint8_t acc = accept_bools[lp];
                if (acc > 0) {
                    const float ppx = in_prev_frame_pixel[lp * 2], ppy = in_prev_frame_pixel[lp * 2 + 1];
                    const int ix = floor_to_int(ppx), iy = floor_to_int(ppy);
                    const float fx = ppx - (float)ix, fy = ppy - (float)iy;
                    const float ofx = 1.0f - fx, ofy = 1.0f - fy;
                    float total = 0.0f;
                    const float wts[4] = {ofx * ofy, fx * ofy, ofx * fy, fx * fy};
                    const int dx[4] = {0, 1, 0, 1}, dy[4] = {0, 0, 1, 1};
                    for (int i = 0; i < 4; ++i) {
                        if (acc & (1 << i)) {
                            total = total + wts[i];
                            const int s = (iy + dy[i]) * g.W + ix + dx[i];
                            for (int c = 0; c < 3; ++c)
                                prev[c] = prev[c] + wts[i] * accumulated_prev_frame[s * 3 + c];
                        }
                    }
                    if (total > 0.0f) {
                        alpha = 1.0f / (float)current_spp[lp];
                        alpha = fmax_cl(alpha, cfg->second_blend_alpha);
                        for (int c = 0; c < 3; ++c) prev[c] = prev[c] / total;
                    }
                }
            }
            const float one_minus = 1.0f - alpha;
            float acc_c[3];
            for (int c = 0; c < 3; ++c) {
                acc_c[c] = alpha * fc[c] + one_minus * prev[c];
                accumulated_frame[lp * 3 + c] = acc_c[c];
            }
            for (int c = 0; c < 3; ++c) {
                // clamp(powr(max(0, albedo * acc), 0.454545f), 0, 1)
                float x = fmax_cl(0.0f, albedo[lp * 3 + c] * acc_c[c]);
                float t = x > 0.0f ? std::pow(x, 0.454545f) : (x == 0.0f ? 0.0f : x);
                t = fmin_cl(fmax_cl(t, 0.0f), 1.0f);
                tone_mapped_frame[lp * 3 + c] = t;
            }
        }
    }
}

void orc_taa(const orc_cfg* cfg, const float* in_prev_frame_pixel, const float* new_frame,
             float* result_frame, const float* prev_frame, int frame_number) {
    Geometry g(cfg);
    const float ta = cfg->taa_blend_alpha;
    const int nt = threads_of(cfg);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int py = 0; py < g.H; ++py) {
        for (int px = 0; px < g.W; ++px) {
            const int lp = py * g.W + px;
            const float* mine = new_frame + lp * 3;
            const float ppx = in_prev_frame_pixel[lp * 2], ppy = in_prev_frame_pixel[lp * 2 + 1];
            const int ix = floor_to_int(ppx), iy = floor_to_int(ppy);
            if (frame_number == 0 || ix < -1 || iy < -1 || ix >= g.W || iy >= g.H) {
                for (int c = 0; c < 3; ++c) result_frame[lp * 3 + c] = mine[c];
                continue;
            }
            float mnb[3] = {INFINITY, INFINITY, INFINITY}, mnc[3] = {INFINITY, INFINITY, INFINITY};
            float mxb[3] = {-INFINITY, -INFINITY, -INFINITY}, mxc[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (int y = -1; y < 2; ++y) {
                for (int x = -1; x < 2; ++x) {
                    const int sx = px + x, sy = py + y;
                    if (sx >= 0 && sy >= 0 && sx < g.W && sy < g.H) {
                        const float* s = new_frame + (sy * g.W + sx) * 3;
                        // RGB_to_YCoCg (bmfr.cl:184-190)
                        const float ycc[3] = {(s[0] * 1.0f + s[1] * 2.0f) + s[2] * 1.0f,
                                              (s[0] * 2.0f + s[1] * 0.0f) + s[2] * -2.0f,
                                              (s[0] * -1.0f + s[1] * 2.0f) + s[2] * -1.0f};
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
            float prev[3] = {0.f, 0.f, 0.f};
            float total = 0.0f;
            const float fx = ppx - (float)ix, fy = ppy - (float)iy;
            const float ofx = 1.0f - fx, ofy = 1.0f - fy;
            auto tap = [&](int sx, int sy, float w) {
                const float* s = prev_frame + (sy * g.W + sx) * 3;
                for (int c = 0; c < 3; ++c) prev[c] = prev[c] + w * s[c];
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
            for (int c = 0; c < 3; ++c) prev[c] = prev[c] / total;
            const float pyc[3] = {(prev[0] * 1.0f + prev[1] * 2.0f) + prev[2] * 1.0f,
                                  (prev[0] * 2.0f + prev[1] * 0.0f) + prev[2] * -2.0f,
                                  (prev[0] * -1.0f + prev[1] * 2.0f) + prev[2] * -1.0f};
            float cl[3];
            for (int c = 0; c < 3; ++c) {
                const float lo = (mnb[c] + mnc[c]) / 2.0f;
                const float hi = (mxb[c] + mxc[c]) / 2.0f;
                cl[c] = fmin_cl(fmax_cl(pyc[c], lo), hi);
            }
            // YCoCg_to_RGB (bmfr.cl:192-198)
            const float rgb[3] = {(cl[0] * 0.25f + cl[1] * 0.25f) + cl[2] * -0.25f,
                                  (cl[0] * 0.25f + cl[1] * 0.0f) + cl[2] * 0.25f,
                                  (cl[0] * 0.25f + cl[1] * -0.25f) + cl[2] * -0.25f};
            const float om = 1.0f - ta;
            for (int c = 0; c < 3; ++c) result_frame[lp * 3 + c] = ta * mine[c] + om * rgb[c];
        }
    }
}

}  // extern "C"
