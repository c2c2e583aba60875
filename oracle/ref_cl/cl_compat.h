// cl_compat.h — TEST INFRASTRUCTURE ONLY.
//
// The OpenCL C 1.2 surface that the reference's kernels (opencl/bmfr.cl) use,
// written as C++ so that g++ compiles that kernel source for the CPU: vector
// types with their component-wise operators, the swizzles the kernels read
// (.xyz of float4, .s048c/.s159d/.s26ae/.s37bf of float16), the built-in
// functions they call, the work-item functions and barriers.  The executor
// (ref_runner.cpp) runs a work-group's work-items as fibers and switches at
// every barrier.
//
// Arithmetic follows the OpenCL C specification where it defines it, and
// otherwise makes the choices the oracle states:
//  * every vector operation rounds component by component (the kernels are
//    compiled with -ffp-contract=off: no fused multiply-add);
//  * dot() is evaluated left to right, ((a.x*b.x + a.y*b.y) + a.z*b.z) + a.w*b.w
//    (the specification leaves the order open);
//  * fmin/fmax/min/max/clamp are the specification's definitions
//    ("y if y < x, else x" and so on, fmin/fmax returning the other operand
//    of a NaN);
//  * vstore_half rounds to nearest even (the default rounding mode);
//  * convert_int2_rtn is floor; NaN and values beyond +-2^30 map to -2^30 /
//    +2^30 (the specification leaves out-of-range conversions undefined);
//  * convert_uchar_sat_rte rounds to nearest even and saturates, NaN to 0;
//  * sqrt is the correctly rounded sqrtf, powr is powf for x >= 0.
#pragma once

#include <cmath>
#include <climits>
#include <cstddef>
#include <cstdint>

namespace clc {

// ---- work-item state, owned by the executor --------------------------------
struct WorkItem {
    size_t global_id[3];
    size_t local_id[3];
    size_t group_id[3];
};
extern thread_local const WorkItem* tl_item;   // the running work-item
void barrier_yield();                          // fiber switch at a barrier

// ---- scalar types -----------------------------------------------------------
typedef unsigned char uchar;
typedef unsigned int uint;
typedef uint16_t half;     // storage only: vload_half / vstore_half

// ---- vectors ----------------------------------------------------------------
struct int2 {
    int x, y;
    int2() = default;
    constexpr int2(int s) : x(s), y(s) {}
    constexpr int2(int a, int b) : x(a), y(b) {}
};
struct int3 {              // result of a float3 relational operator: -1 / 0
    int x, y, z;
};
struct float2 {
    float x, y;
    float2() = default;
    constexpr float2(float s) : x(s), y(s) {}
    constexpr float2(float a, float b) : x(a), y(b) {}
};
struct alignas(16) float3 {
    float x, y, z;
    float3() = default;
    constexpr float3(float s) : x(s), y(s), z(s) {}
    constexpr float3(float a, float b, float c) : x(a), y(b), z(c) {}
};
struct float4;

// The .xyz swizzle of float4: a member of float4's union that reads and
// writes the first three components in place.
struct SwizzleXYZ {
    float v[4];
    operator float3() const { return float3(v[0], v[1], v[2]); }
    SwizzleXYZ& operator=(const float3& a) {
        v[0] = a.x; v[1] = a.y; v[2] = a.z;
        return *this;
    }
};

struct alignas(16) float4 {
    union {
        struct { float x, y, z, w; };
        SwizzleXYZ xyz;
    };
    float4() = default;
    constexpr float4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
};

// Four-component swizzles of float16 (.sABCD, hexadecimal component indices).
template <int A, int B, int C, int D>
struct Swizzle16x4 {
    float v[16];
    operator float4() const { return float4(v[A], v[B], v[C], v[D]); }
};

struct alignas(64) float16 {
    union {
        float s[16];
        Swizzle16x4<0, 4, 8, 12> s048c;
        Swizzle16x4<1, 5, 9, 13> s159d;
        Swizzle16x4<2, 6, 10, 14> s26ae;
        Swizzle16x4<3, 7, 11, 15> s37bf;
    };
};

// ---- component-wise operators ------------------------------------------------
inline int2 operator+(int2 a, int2 b) { return int2(a.x + b.x, a.y + b.y); }
inline int2 operator-(int2 a, int2 b) { return int2(a.x - b.x, a.y - b.y); }

inline float2 operator+(float2 a, float2 b) { return float2(a.x + b.x, a.y + b.y); }
inline float2 operator-(float2 a, float2 b) { return float2(a.x - b.x, a.y - b.y); }
inline float2 operator*(float2 a, float2 b) { return float2(a.x * b.x, a.y * b.y); }
inline float2 operator/(float2 a, float2 b) { return float2(a.x / b.x, a.y / b.y); }
inline float2& operator+=(float2& a, float2 b) { return a = a + b; }
inline float2& operator-=(float2& a, float2 b) { return a = a - b; }
inline float2& operator*=(float2& a, float2 b) { return a = a * b; }
inline float2& operator/=(float2& a, float2 b) { return a = a / b; }

inline float3 operator+(float3 a, float3 b) { return float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a, float3 b) { return float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator*(float3 a, float3 b) { return float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator/(float3 a, float3 b) { return float3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline float3& operator+=(float3& a, float3 b) { return a = a + b; }
inline float3& operator-=(float3& a, float3 b) { return a = a - b; }
inline float3& operator*=(float3& a, float3 b) { return a = a * b; }
inline float3& operator/=(float3& a, float3 b) { return a = a / b; }
inline int3 operator<(float3 a, float3 b) {
    return int3{a.x < b.x ? -1 : 0, a.y < b.y ? -1 : 0, a.z < b.z ? -1 : 0};
}

// `mask ? a : b` of OpenCL C for vectors: per component, a where the mask's
// most significant bit is set, else b.
inline float3 clc_vselect(int3 m, float3 a, float3 b) {
    return float3(m.x < 0 ? a.x : b.x, m.y < 0 ? a.y : b.y, m.z < 0 ? a.z : b.z);
}

// ---- work-item functions and synchronisation -------------------------------
inline size_t get_global_id(uint d) { return tl_item->global_id[d]; }
inline size_t get_local_id(uint d) { return tl_item->local_id[d]; }
inline size_t get_group_id(uint d) { return tl_item->group_id[d]; }

#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2
inline void barrier(int) { barrier_yield(); }

// ---- built-in functions -------------------------------------------------------
inline float dot(float3 a, float3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline float dot(float4 a, float4 b) { return ((a.x * b.x + a.y * b.y) + a.z * b.z) + a.w * b.w; }

inline float fmin(float x, float y) {
    if (std::isnan(x)) return y;
    if (std::isnan(y)) return x;
    return y < x ? y : x;
}
inline float fmax(float x, float y) {
    if (std::isnan(x)) return y;
    if (std::isnan(y)) return x;
    return x < y ? y : x;
}
inline float3 fmin(float3 a, float3 b) { return float3(fmin(a.x, b.x), fmin(a.y, b.y), fmin(a.z, b.z)); }
inline float3 fmax(float3 a, float3 b) { return float3(fmax(a.x, b.x), fmax(a.y, b.y), fmax(a.z, b.z)); }

inline int min(int x, int y) { return y < x ? y : x; }
inline int max(int x, int y) { return x < y ? y : x; }
inline float min(float x, float y) { return y < x ? y : x; }
inline float max(float x, float y) { return x < y ? y : x; }
inline float3 max(float3 a, float3 b) { return float3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }

inline float3 clamp(float3 x, float3 lo, float3 hi) { return fmin(fmax(x, lo), hi); }

inline float sqrt(float x) { return std::sqrt(x); }
inline float fabs(float x) { return std::fabs(x); }
inline int isnan(float x) { return std::isnan(x) ? 1 : 0; }

inline float powr1(float x, float y) { return std::pow(x, y); }
inline float3 powr(float3 x, float3 y) { return float3(powr1(x.x, y.x), powr1(x.y, y.y), powr1(x.z, y.z)); }

inline float convert_float(unsigned int v) { return (float)v; }
inline float convert_float(int v) { return (float)v; }
inline float convert_float(unsigned char v) { return (float)v; }
inline float convert_float(float v) { return v; }
inline float convert_float(double v) { return (float)v; }
inline float2 convert_float2(int2 v) { return float2((float)v.x, (float)v.y); }

inline int clc_floor_int(float v) {
    if (std::isnan(v)) return -(1 << 30);
    const float f = std::floor(v);
    if (f < -1073741824.0f) return -(1 << 30);
    if (f > 1073741824.0f) return 1 << 30;
    return (int)f;
}
inline int2 convert_int2_rtn(float2 v) { return int2(clc_floor_int(v.x), clc_floor_int(v.y)); }

inline uchar convert_uchar_sat_rte(float v) {
    if (std::isnan(v)) return 0;
    const float r = std::nearbyint(v);    // the default rounding mode: nearest even
    if (r <= 0.0f) return 0;
    if (r >= 255.0f) return 255;
    return (uchar)r;
}

inline float vload_half(size_t i, const half* p) {
    _Float16 h;
    __builtin_memcpy(&h, p + i, 2);
    return (float)h;
}
inline void vstore_half(float v, size_t i, half* p) {
    const _Float16 h = (_Float16)v;        // round to nearest even
    __builtin_memcpy(p + i, &h, 2);
}

}  // namespace clc

// ---- address-space and function qualifiers ------------------------------------
// (defined after every system header, so they touch only the kernel source)
#define __kernel
#define __global
#define __local
#define local
#define __constant const
#define restrict __restrict__
#define CLC_KERNEL_LOCAL static thread_local
