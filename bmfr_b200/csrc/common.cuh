// common.cuh — constants, geometry and exact-arithmetic helpers shared by the
// sm_100a kernels of the BMFR pipeline.
//
// The library is compiled with -fmad=false: no multiply and add is contracted
// into a fused multiply-add unless a kernel asks for it explicitly, so every
// float expression is rounded operation by operation in the order written —
// the order of the reference's expressions (opencl/bmfr.cl).  Division and
// square root are IEEE round-to-nearest (nvcc's default -prec-div/-prec-sqrt).
#pragma once

#include <cstdint>
#include <cuda_fp16.h>

namespace bmfr {

constexpr int kBlockEdge = 32;       // BLOCK_EDGE_LENGTH (bmfr.cpp:104)
constexpr int kBlockPixels = 1024;   // BLOCK_PIXELS (bmfr.cpp:105)
constexpr int kLocal = 256;          // fitter work-group (bmfr.cpp:116)
constexpr int kBuffers = 13;         // BUFFER_COUNT
constexpr int kFeatures = 10;        // BUFFER_COUNT - 3
constexpr int kNotScaled = 4;        // FEATURES_NOT_SCALED
constexpr int kScaled = 6;           // FEATURES_SCALED
constexpr int kREdge = 11;           // R_EDGE

// BLOCK_OFFSETS (bmfr.cl:267-285): per-frame jitter of the block grid.
static __constant__ int2 c_block_offsets[16] = {
    {-14, -14}, {4, -6}, {-8, 14}, {8, 0}, {-10, -8}, {2, 12}, {12, -12}, {-10, 0},
    {12, 14}, {-8, -16}, {6, 6}, {-2, -2}, {6, -14}, {-16, 12}, {14, -4}, {-6, 4}};

// Image, workset and margin sizes of one stream (bmfr.cpp:104-118).
struct Geometry {
    int W, H;          // IMAGE_WIDTH/HEIGHT
    int MW, MH;        // WORKSET_WITH_MARGINS_WIDTH/HEIGHT
    int MWb, MHb;      // margin grid in blocks
    int blocks;        // MWb * MHb
};

inline Geometry make_geometry(int W, int H) {
    Geometry g;
    g.W = W;
    g.H = H;
    const int ww = kBlockEdge * ((W + kBlockEdge - 1) / kBlockEdge);
    const int wh = kBlockEdge * ((H + kBlockEdge - 1) / kBlockEdge);
    g.MW = ww + kBlockEdge;
    g.MH = wh + kBlockEdge;
    g.MWb = g.MW / kBlockEdge;
    g.MHb = g.MH / kBlockEdge;
    g.blocks = g.MWb * g.MHb;
    return g;
}

// Per-frame scalars of accumulate_noisy_data (bmfr.cl:306-308 plus the -D
// limits and blend factor).
struct AccumArgs {
    float m[16];              // prev_frame_camera_matrix (float16 argument)
    float off_x, off_y;       // pixel_offset
    float pos_lim2, nrm_lim2; // POSITION/NORMAL_LIMIT_SQUARED
    float blend_alpha;        // BLEND_ALPHA
    int frame;
    int use_half;             // tmp_data element type
};

// NOISE_AMOUNT * 2 as an unevaluated sum of two floats (hi + lo), so that
// value + NOISE_AMOUNT * 2 * r, which the reference forms in double because
// NOISE_AMOUNT is a double literal (bmfr.cpp:58, bmfr.cl:179), is rounded
// once to float without double arithmetic on the device.
struct NoiseConst {
    float hi, lo;
    float neg_zero;   // -0.0f, known only at run time: the addend of the fitter's products (rmul2)
};

// OpenCL's fmin/fmax (and max(x, y) for the operands the kernels give it):
// y if y < x (x < y), else x; the other operand when x is NaN.  A NaN
// reaches them in taa when every bilinear weight of the history is zero
// (bmfr.cl:939: 0/0), and the clamp then returns the bound.
__device__ __forceinline__ float fmin_cl(float x, float y) { return (y < x || x != x) ? y : x; }
__device__ __forceinline__ float fmax_cl(float x, float y) { return (x < y || x != x) ? y : x; }

// mirror (bmfr.cl:209-216): valid for indices at most one size out of range.
__device__ __forceinline__ int mirror(int i, int n) {
    if (i < 0) return -i - 1;
    if (i >= n) return 2 * n - i - 1;
    return i;
}

// Programmatic dependent launch.  The pipeline's kernels are launched with
// programmatic stream serialization (launch_chained), so a kernel's launch
// is processed while the kernel before it in the stream drains; before it
// touches memory it waits here for that kernel's completion and memory
// flush, which keeps exactly the ordering of a plain stream.  Dependents
// are released implicitly as CTAs exit (no early trigger: released early,
// waiting CTAs would take the SM slots that multi-wave grids still need).
// Without the launch attribute this is a no-op.
__device__ __forceinline__ void await_previous_kernel() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// convert_int_rtn with defined results: NaN and magnitudes beyond 2^30 map to
// +-2^30, outside every image.
__device__ __forceinline__ int floor_to_int(float v) {
    if (!(v == v)) return -(1 << 30);
    const float f = floorf(v);
    if (f < -1073741824.0f) return -(1 << 30);
    if (f > 1073741824.0f) return 1 << 30;
    return (int)f;
}

// random() (bmfr.cl:162-171): a 32-bit integer hash mapped to [0, 1].
__device__ __forceinline__ float hash_random(uint32_t a) {
    a = (a + 0x7ed55d16u) + (a << 12);
    a = (a ^ 0xc761c23cu) ^ (a >> 19);
    a = (a + 0x165667b1u) + (a << 5);
    a = (a + 0xd3a2646cu) ^ (a << 9);
    a = (a + 0xfd7046c5u) + (a << 3);
    a = (a ^ 0xb55a4f09u) ^ (a >> 16);
    return __uint2float_rn(a) / 4294967296.0f;   // convert_float(UINT_MAX) = 2^32
}

// add_random (bmfr.cl:173-182): value + NOISE_AMOUNT*2*(random(i) - 0.5),
// rounded once to float.  The product c*r (c = hi + lo) is formed exactly
// enough with fma error terms (Dekker/Ogita-Rump-Oishi two-product and
// two-sum), then the three-term sum is rounded once.
__device__ __forceinline__ float add_noise(float value, uint32_t index, NoiseConst c) {
    const float r = hash_random(index) - 0.5f;
    const float p = c.hi * r;
    const float pe = __fmaf_rn(c.hi, r, -p);          // exact error of c.hi*r
    const float pl = __fmaf_rn(c.lo, r, pe);          // + c.lo*r
    const float s = value + p;                        // two-sum(value, p)
    const float bv = s - value;
    const float se = (value - (s - bv)) + (p - bv);
    return s + (se + pl);
}

__device__ __forceinline__ uint32_t noise_index(int id, int sub_vector, int feature, int frame) {
    return (uint32_t)id + (uint32_t)sub_vector * (uint32_t)kLocal +
           (uint32_t)feature * (uint32_t)kBlockPixels +
           (uint32_t)frame * (uint32_t)(kBuffers * kBlockPixels);
}

// scale (bmfr.cl:200-205).
__device__ __forceinline__ float scale(float v, float mn, float mx) {
    if (fabsf(mx - mn) > 1.0f) return (v - mn) / (mx - mn);
    return v - mn;
}

__device__ __forceinline__ float round_half(float v) {
    return __half2float(__float2half_rn(v));
}

// Store of one tmp_data value, binary16 or float32 (bmfr.cl:255-265, 468-475).
__device__ __forceinline__ void store_feature(void* tmp, size_t i, float v, bool half_tmp) {
    if (v != v) v = 0.0f;
    if (half_tmp) {
        v = fmaxf(fminf(v, 65504.0f), -65504.0f);
        reinterpret_cast<__half*>(tmp)[i] = __float2half_rn(v);
    } else {
        reinterpret_cast<float*>(tmp)[i] = v;
    }
}

__device__ __forceinline__ void hist_store(float* p, int i, float3 v) {
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}
__device__ __forceinline__ void hist_store(__half* p, int i, float3 v) {
    p[3 * i] = __float2half_rn(v.x);
    p[3 * i + 1] = __float2half_rn(v.y);
    p[3 * i + 2] = __float2half_rn(v.z);
}

__device__ __forceinline__ float3 load3(const float* p, int i) {
    return make_float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}
__device__ __forceinline__ void store3(float* p, int i, float3 v) {
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}

}  // namespace bmfr
