// fit_block.cuh — the per-block least-squares fit of BMFR (opencl/bmfr.cl:
// 490-700) as a device routine for one 256-thread CTA, shared by the
// standalone fitter kernel and the fused accumulate+fit kernel.
//
// Layout.  Each thread is one of the reference's 256 work-items and owns the
// same four pixels of the 32x32 block (rows id, id+256, id+512, id+768 of the
// 1024x13 matrix).  The block stays in registers through the min/max
// scaling, the ten Householder reflections and their updates, as binary16
// pairs when the reference rounds every in-place store to half
// (bmfr.cl:540, 651) — the packed conversion is that rounding — and as
// floats otherwise.  tmp_data is never written back.  Work-item ids are
// assigned to lanes as
//     id = 8*warp + (lane & 7) + 64*(lane >> 3)
// so that the first stage of the reference's reduction tree (ids i, i+64,
// i+128, i+192, bmfr.cl:32-33) sits inside one warp and runs on shuffles.
//
// Reductions.  block_reduce (min/max), block_sum_dots and block_sum1_all
// evaluate parallel_reduction_sum/min/max (bmfr.cl:25-87) over exactly the
// same tree, so the sums round exactly as the reference's do.  The batched
// forms reduce up to 12 independent values behind one pair of barriers: the
// twelve min/max values of the scaling step, and per column the up to twelve
// dot products, which are independent once the Householder vector is known.
// A column costs the norm (one barrier) and the dots (two) where the
// reference spends three barriers per dot product.
//
// Columns run in a loop; each column's update writes later column k into
// tile slot k - 1, so the tile moves down by one column as it is updated and
// every index into it is a compile-time constant.
//
// Division.  The rank-one update divides by the column's |u|^2, which is the
// same for the whole block.  Its correctly rounded reciprocal is formed once
// and every quotient is taken with Markstein's correction step
// (q = a*y; r = fma(-q, b, a); q' = fma(r, y, q)), which returns the
// correctly rounded a/b while numerator, divisor and quotient stay normal;
// operands outside the ranges that guarantee this take a true division.
//
// The colour columns' own reflections (columns 10..12, bmfr.cl:549 with
// col_limited = 10) only change rows >= 10, which neither the back
// substitution nor the weights read (bmfr.cl:660-699), so they are skipped.
#pragma once

#include "common.cuh"

namespace bmfr {

// Row stride of FitterSmem::part: 64 first-stage sums per value plus three
// floats of padding, so that the 8-lane groups storing values i and i + 6
// (or i + 3) and the groups reading values v and v + 8 fall on distinct banks.
constexpr int kPartStride = 67;

struct FitterSmem {
    float part[13 * kPartStride];   // first-stage partial sums of the batched values
    float out[16];         // reduction results
    float ucl;             // u[col] broadcast from its owner
    int status;            // nonzero: a bounded wait ran out
    float Rm[10][10];      // R of the ten feature columns: Rm[x][y], y <= x
    float rhs[10][3];      // rows 0..9 of the three colour columns
    float part1[64];       // first-stage sums of block_sum1_all
    float gram[88];        // CholeskyQR2: the Gram entries of a pass, summed over the warps
    float rowc[13];        // the precision form: row `col` of every column
    float inv1[10];        // CholeskyQR2: reciprocals of R1's and R2's diagonals,
    float inv2[10];        //   and the diagonal of the Gram matrix being factored
    float diag[10];
};

// How the block's least-squares system is solved.
enum FitMethod : int {
    kFitReference = 0,     // the reference's Householder sequence and rounding
    kFitCholQR2 = 1,       // precision form: CholeskyQR2 in FP32
    kFitHouseholder32 = 2  // precision form: the Householder sequence in FP32
};

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int work_item_id() {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    return 8 * warp + (lane & 7) + 64 * (lane >> 3);
}

template <int OP>
__device__ __forceinline__ float rop(float a, float b) {
    if (OP == 0) return a + b;
    if (OP == 1) return fmin_cl(a, b);
    return fmax_cl(a, b);
}

// Batched work-group min/max reduction of n <= VMAX values per thread
// (parallel_reduction_min/max, bmfr.cl:45-87).  Values [0, split) use OP_A,
// [split, n) use OP_B (1 min, 2 max); results in sm.out.
template <int VMAX, int OP_A, int OP_B>
__device__ __forceinline__ void block_reduce(const float (&v)[VMAX], int n, int split, FitterSmem& sm) {
    static_assert(OP_A != 0 && OP_B != 0, "sums go through block_sum_dots or block_sum1_all");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < VMAX; ++i) {
        if (i < n) {
            const float a = v[i];
            const float b = __shfl_down_sync(kFull, a, 8);
            const float c = __shfl_down_sync(kFull, a, 16);
            const float d = __shfl_down_sync(kFull, a, 24);
            const int op = i < split ? OP_A : OP_B;
            float s1;
            if (op == 1) s1 = fmin_cl(fmin_cl(fmin_cl(a, b), c), d);    // bmfr.cl:52-53
            else s1 = fmax_cl(fmax_cl(fmax_cl(a, b), c), d);            // bmfr.cl:74-75
            if (lane < 8) sm.part[i * kPartStride + 8 * warp + lane] = s1;
        }
    }
    __syncthreads();
    // Stages 2 and 3: value vi is finished by the 8-lane group `lane >> 3` of
    // warp vi % 8; lane j of the group forms the j-th second-stage value
    // (bmfr.cl:56-58), lane 0 of the group the result (bmfr.cl:60-63).
    const int vi = warp + 8 * (lane >> 3);
    const int j = lane & 7;
    const int op = vi < split ? OP_A : OP_B;
    float s2 = 0.0f;
    if (vi < n) {
        const float* p = sm.part + vi * kPartStride + j;
        float acc = p[0];
#pragma unroll
        for (int m = 1; m < 8; ++m) acc = op == 1 ? fmin_cl(acc, p[8 * m]) : fmax_cl(acc, p[8 * m]);
        s2 = acc;
    }
    if (warp < n) {   // warp-uniform: warps without a value skip
        float r = __shfl_sync(kFull, s2, 0, 8);
#pragma unroll
        for (int m = 1; m < 8; ++m) {
            const float x = __shfl_sync(kFull, s2, m, 8);
            r = op == 1 ? fmin_cl(r, x) : fmax_cl(r, x);
        }
        if (vi < n && j == 0) sm.out[vi] = r;
    }
    __syncthreads();
}

// parallel_reduction_sum (bmfr.cl:25-43) of the column step's n <= VMAX dot
// products; results in sm.out.  NMIN is a compile-time lower bound on n: the
// guards of the values below it vanish.  Returns, from the closing barrier,
// whether any sum lies outside {0} and [2^-32, 2^30], the range in which the
// update's quotients take Markstein's correction.
//
// Stage 1 (bmfr.cl:33) is a transposing exchange: the lanes of ids i+64 and
// i+128 (groups 1 and 2) swap half of their values and form b + c, the lanes
// of ids i and i+192 (groups 0 and 3) swap the other half and each receive
// b + c from their neighbour group, so group 0 finishes values [0, H) and
// group 3 values [H, 2H) as a + ((b + c) + d): one shuffle per value instead
// of three.  Stages 2 and 3 as in block_reduce.
template <int VMAX, int NMIN>
__device__ __forceinline__ bool block_sum_dots(const float (&v)[VMAX], int n, FitterSmem& sm) {
    constexpr int H = (VMAX + 1) / 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 3;
    const bool low = g < 2;   // groups 0 and 1 keep values [0, H), 2 and 3 values [H, 2H)
    float* dst = sm.part + (g == 0 ? 0 : H * kPartStride) + 8 * warp + (lane & 7);
#pragma unroll
    for (int i = 0; i < H; ++i) {
        if (i < NMIN || i < n) {
            const float x = v[i], y = H + i < VMAX ? v[H + i] : 0.0f;
            const float keep = low ? x : y;
            const float got = __shfl_xor_sync(kFull, low ? y : x, 24);
            const float bc = keep + got;                            // groups 1 and 2: b + c
            const float bc_in = __shfl_xor_sync(kFull, bc, 8);      // groups 0 and 3 receive it
            const float a = g == 0 ? keep : got, d = g == 0 ? got : keep;
            const float s1 = a + (bc_in + d);
            if (g == 0 || (g == 3 && (H + i < NMIN || H + i < n))) dst[i * kPartStride] = s1;
        }
    }
    __syncthreads();
    // Stage 2 (bmfr.cl:35-37): value vi is finished by the 8-lane group
    // `lane >> 3` of warp vi % 8; lane j of the group forms sum_vec[j].
    const int vi = warp + 8 * g;
    const int j = lane & 7;
    float s2 = 0.0f;
    if (vi < n) {
        const float* p = sm.part + vi * kPartStride + j;
        float acc = p[8];
#pragma unroll
        for (int m = 2; m < 8; ++m) acc = acc + p[8 * m];
        s2 = p[0] + acc;
    }
    // Stage 3 (bmfr.cl:39-42): sum_vec[0] + ... + sum_vec[7], left to right,
    // by lane 0 of the group from its lanes' values on shuffles.
    bool out_of_range = false;
    if (warp < n) {   // warp-uniform: warps without a value skip
        float r = __shfl_sync(kFull, s2, 0, 8);
#pragma unroll
        for (int m = 1; m < 8; ++m) r = r + __shfl_sync(kFull, s2, m, 8);
        if (vi < n && j == 0) {
            sm.out[vi] = r;
            const float ar = fabsf(r);
            out_of_range = !(ar == 0.0f || (ar >= 0x1p-32f && ar <= 0x1p30f));
        }
    }
    return __syncthreads_or(out_of_range) != 0;
}

// parallel_reduction_sum (bmfr.cl:25-43) of one value per thread, finished by
// every warp: stage 1 inside each warp on shuffles (ids i, i+64, i+128,
// i+192), one barrier, then each warp reads the 64 first-stage sums and runs
// stages 2 and 3 itself in the reference's order, so the sum reaches every
// thread without a second barrier or a broadcast through shared memory.
// part1 is rewritten only by the next call, and block_sum_dots' barriers
// separate consecutive calls in the column loop, so no warp can overwrite
// sums another warp is still reading.
__device__ __forceinline__ float block_sum1_all(float v, FitterSmem& sm) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float b = __shfl_down_sync(kFull, v, 8);
    const float c = __shfl_down_sync(kFull, v, 16);
    const float d = __shfl_down_sync(kFull, v, 24);
    const float s1 = v + ((b + c) + d);   // bmfr.cl:33
    if (lane < 8) sm.part1[8 * warp + lane] = s1;
    __syncthreads();
    // Stage 2 (bmfr.cl:35-37): lane j < 8 forms sum_vec[j].
    float s2 = 0.0f;
    if (lane < 8) {
        const float* p = sm.part1 + lane;
        float acc = p[8];
#pragma unroll
        for (int m = 2; m < 8; ++m) acc = acc + p[8 * m];
        s2 = p[0] + acc;
    }
    // Stage 3 (bmfr.cl:39-42): sum_vec[0] + ... + sum_vec[7], left to right.
    float r = __shfl_sync(kFull, s2, 0);
#pragma unroll
    for (int k = 1; k < 8; ++k) r = r + __shfl_sync(kFull, s2, k);
    return r;
}

// The block as held by one thread: four rows of the 13 columns.
template <bool HALF>
struct Tile;

template <>
struct Tile<true> {   // binary16 storage: every store rounds to nearest even
    __half2 h[kBuffers][2];
    __device__ __forceinline__ float2 get2(int k, int p) const { return __half22float2(h[k][p]); }
    __device__ __forceinline__ void set2(int k, int p, float a, float b) { h[k][p] = __floats2half2_rn(a, b); }
};

template <>
struct Tile<false> {   // float storage: no intermediate rounding; rows (q0,q1) and (q2,q3) paired
    float2 p[kBuffers][2];
    __device__ __forceinline__ float2 get2(int k, int h) const { return p[k][h]; }
    __device__ __forceinline__ void set2(int k, int h, float a, float b) { p[k][h] = make_float2(a, b); }
    __device__ __forceinline__ float get1(int k, int q) const { return (q & 1) ? p[k][q >> 1].y : p[k][q >> 1].x; }
    __device__ __forceinline__ void set1(int k, int q, float v) {
        if (q & 1) p[k][q >> 1].y = v;
        else p[k][q >> 1].x = v;
    }
};

// value + NOISE_AMOUNT*2*r with r = random(i) - 0.5 already formed
// (bmfr.cl:173-182), rounded once (see add_noise in common.cuh).
__device__ __forceinline__ float add_noise_r(float value, float r, NoiseConst c) {
    const float p = c.hi * r;
    const float pe = __fmaf_rn(c.hi, r, -p);
    const float pl = __fmaf_rn(c.lo, r, pe);
    const float s = value + p;
    const float bv = s - value;
    const float se = (value - (s - bv)) + (p - bv);
    return s + (se + pl);
}

// True division, kept out of line so that the rare slow case costs no code
// at every call site.
static __device__ __noinline__ float div_slow(float a, float b) { return a / b; }

// scale() (bmfr.cl:200-205) with the quotient taken by Markstein's
// correction when numerator and divisor keep it normal.
__device__ __forceinline__ float scale_by(float v, float mn, float mx) {
    const float d = mx - mn;
    const float num = v - mn;
    if (!(fabsf(d) > 1.0f)) return num;
    const float an = fabsf(num);
    if (d <= 0x1p60f && (an == 0.0f || (an >= 0x1p-64f && an <= 0x1p60f))) {
        const float y = __frcp_rn(d);
        const float q0 = num * y;
        const float r = __fmaf_rn(-q0, d, num);
        return -__fmaf_rn(-r, y, -q0);
    }
    return div_slow(num, d);
}

// Table of the fitter's feature noise r = random(i) - 0.5 (bmfr.cl:179-181)
// for features 1..9, laid out [feature-1][row group q][thread] so that each
// thread reads its own four rows coalesced.  It does not involve the block
// index, so one table serves every block of a frame; it lives in shared
// memory (standalone fitter) or global memory (frame pipeline).
constexpr int kNoiseTableFloats = (kFeatures - 1) * 4 * kLocal;

__device__ __forceinline__ float noise_table_value(int entry, int frame) {
    const int tx = entry % kLocal, fq = entry / kLocal;   // fq = (fb-1)*4 + q
    const int fb = fq / 4 + 1, q = fq % 4;
    const int warp = tx >> 5, lane = tx & 31;
    const int id = 8 * warp + (lane & 7) + 64 * (lane >> 3);
    return hash_random(noise_index(id, q, fb, frame)) - 0.5f;
}

__device__ __forceinline__ void fill_noise_table(float* table, int frame) {
    for (int e = threadIdx.x; e < kNoiseTableFloats; e += kLocal) table[e] = noise_table_value(e, frame);
}

// Packed FP32 (sm_100 FADD2/FMUL2/FFMA2): two independent IEEE operations,
// each rounded exactly as the scalar form, in one instruction.
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// Products that must round on their own.  A packed multiply whose result
// feeds a packed add is fused into one packed fused multiply-add by the
// compiler, even when written in PTX with an explicit rounding mode
// (measured: the reference-arithmetic fitter then differed from the
// reference in the last bits of most weights with float32 tmp_data).  So the
// product is a fused multiply-add with the addend nz = -0.0f, which the
// caller reads at run time (NoiseConst::neg_zero): RN(a*b + -0) is RN(a*b)
// with its sign of zero, and an FMA cannot be fused into the add it feeds.
__device__ __forceinline__ float2 rmul2(float2 a, float2 b, float nz) { return __ffma2_rn(a, b, make_float2(nz, nz)); }
// RN(a*b + c) for binary16 a, b and a float c (fma.f32.f16): a*b is exact
// in float, so this is RN(c + RN(a*b)), the reference's float multiply-add.
__device__ __forceinline__ float fma_h(__half a, __half b, float c) {
    float d;
    asm("fma.rn.f32.f16 %0, %1, %2, %3;" : "=f"(d)
        : "h"(__half_as_ushort(a)), "h"(__half_as_ushort(b)), "f"(c));
    return d;
}
// RN(a + c) for a binary16 a and a float c: the conversion of a is exact, so
// this is the float addition of the reference, in one instruction.
__device__ __forceinline__ float add_f32_h(__half a, float c) {
    float d;
    asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(d) : "h"(__half_as_ushort(a)), "f"(c));
    return d;
}
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }

// add_noise_r on two values at once.
__device__ __forceinline__ float2 add_noise_r2(float2 v, float2 r, NoiseConst c) {
    const float2 hi = dup2(c.hi), lo = dup2(c.lo);
    const float2 p = rmul2(hi, r, c.neg_zero);
    const float2 pe = fma2(hi, r, neg2(p));
    const float2 pl = fma2(lo, r, pe);
    const float2 sm = add2(v, p);
    const float2 bv = add2(sm, neg2(v));
    const float2 se = add2(add2(v, neg2(add2(sm, neg2(bv)))), add2(p, neg2(bv)));
    return add2(sm, add2(se, pl));
}

// Column k of the tile as two float pairs (rows q0,q1 and q2,q3), with the
// first column's noise added to features 1..9 (bmfr.cl:625-627).
template <bool HALF, bool NOISE>
__device__ __forceinline__ void load_column(const Tile<HALF>& t, int k, int fb, const float* __restrict__ noise,
                                            NoiseConst nc, float2& a01, float2& a23) {
    a01 = t.get2(k, 0);
    a23 = t.get2(k, 1);
    if (NOISE && fb < kFeatures) {
        const float* r = noise + (fb - 1) * 4 * kLocal + threadIdx.x;
        a01 = add_noise_r2(a01, make_float2(r[0], r[kLocal]), nc);
        a23 = add_noise_r2(a23, make_float2(r[2 * kLocal], r[3 * kLocal]), nc);
    }
}

// One Householder column (bmfr.cl:549-655) on tile column 0; later columns
// are tile columns 1..V, and the update leaves later column k in tile
// column k - 1, ready for the next column step (the slots beyond V hold
// columns already finished and are never read again).  NOISE: the first
// column, whose dot products read features 1..9 with noise added
// (bmfr.cl:625-627).
// VS: column slots the loops visit (a compile-time bound >= the V later
// columns): the late columns take a shorter instance.  VMIN: a compile-time
// bound <= V, so that the slots below it are visited without a guard.
template <bool HALF, bool NOISE, int VS = 12, int VMIN = 0>
__device__ __forceinline__ void qr_column(Tile<HALF>& t, int col, int id, const float* __restrict__ noise,
                                          NoiseConst nc, FitterSmem& sm) {
    const int V = kBuffers - 1 - col;
    const float2 c01 = t.get2(0, 0), c23 = t.get2(0, 1);
    // Norm of rows >= col+1 (bmfr.cl:553-569); only row id (q = 0) can be above.
    float nv[1];
    {
        float s = 0.0f;
        if (id >= col + 1) s = s + c01.x * c01.x;
        s = s + c01.y * c01.y;
        s = s + c23.x * c23.x;
        s = s + c23.y * c23.y;
        nv[0] = s;
    }
    if (id == col) sm.ucl = c01.x;   // read after block_sum1_all's barrier
    const float norm2 = block_sum1_all(nv[0], sm);
    const float ucl = sm.ucl;
    // Work-item col's step (bmfr.cl:580-588), evaluated by every thread.
    const float vl = sqrtf(norm2 + ucl * ucl);
    const float ucl_new = ucl - vl;
    const float uls = norm2 + ucl_new * ucl_new;
    if (id < col) sm.Rm[col][id] = c01.x;
    if (id == col) sm.Rm[col][col] = vl;
    const float u0 = id == col ? ucl_new : c01.x;
    const bool row0 = id >= col;
    // Rows below the column (only row id can be) take no part in the dot:
    // 0 + a*0 leaves the reference's partial sum 0 unchanged.
    const float2 uq0 = dup2(row0 ? u0 : 0.0f), uq1 = dup2(c01.y), uq2 = dup2(c23.x), uq3 = dup2(c23.y);

    // Dot products with the later columns (bmfr.cl:606-638): 0 + p0 + p1 +
    // p2 + p3 in the reference's order for rows q0..q3.
    float d[VS];
    if constexpr (HALF && !NOISE) {
        // Row q0 first, as a float product for every thread: the row `col`
        // of one thread has the float u = ucl - vl, and a branch for that
        // thread alone held its warp back at the next barrier (every warp
        // doing the float products measured 4 % faster).  For the other
        // rows a binary16 a times a binary16 u is exact in float, so there
        // 0 + RN(a*u) is the same value the mixed FMA below would give.
        const __half u1 = __high2half(t.h[0][0]), u2 = __low2half(t.h[0][1]), u3 = __high2half(t.h[0][1]);
#pragma unroll
        for (int i = 0; i < VS; i += 2) {
            d[i] = d[i + 1] = 0.0f;
            if (i < VMIN || i < V) {
                const float2 a0 = make_float2(__low2float(t.h[i + 1][0]), __low2float(t.h[i + 2][0]));
                const float2 s = add2(dup2(0.0f), rmul2(a0, uq0, nc.neg_zero));
                d[i] = s.x;
                d[i + 1] = s.y;
            }
        }
        // Rows q1..q3: a binary16 product is exact in float, so s + a*u
        // rounds once either way and is one mixed-precision FMA.
#pragma unroll
        for (int i = 0; i < VS; ++i) {
            if (i < VMIN || i < V) {
                float s = fma_h(__high2half(t.h[i + 1][0]), u1, d[i]);
                s = fma_h(__low2half(t.h[i + 1][1]), u2, s);
                d[i] = fma_h(__high2half(t.h[i + 1][1]), u3, s);
            }
        }
    } else {
        // Two columns at a time in packed lanes; each lane keeps the order.
#pragma unroll
        for (int i = 0; i < VS; i += 2) {
            d[i] = d[i + 1] = 0.0f;
            if (i < VMIN || i < V) {
                float2 a01, a23, b01, b23;
                load_column<HALF, NOISE>(t, i + 1, i + 1, noise, nc, a01, a23);
                load_column<HALF, NOISE>(t, i + 2, i + 2, noise, nc, b01, b23);
                float2 s = add2(dup2(0.0f), rmul2(make_float2(a01.x, b01.x), uq0, nc.neg_zero));
                s = add2(s, rmul2(make_float2(a01.y, b01.y), uq1, nc.neg_zero));
                s = add2(s, rmul2(make_float2(a23.x, b23.x), uq2, nc.neg_zero));
                s = add2(s, rmul2(make_float2(a23.y, b23.y), uq3, nc.neg_zero));
                d[i] = s.x;
                d[i + 1] = s.y;
            }
        }
    }
    const bool dots_out = block_sum_dots<VS, VMIN>(d, V, sm);

    // Rank-one update, rounded at the reference's store (bmfr.cl:640-652).
    // Quotients take Markstein's correction when every operand is in range:
    // |u| and |dot| within [2^-32, 2^30] (or zero) and |u|^2 within 2^+-60
    // keep numerator and quotient normal.  a - RN(num/uls) is formed as
    // a + fma(-r, y, -q0), which keeps the sign of zero quotients exact.
    const float y = __frcp_rn(uls);
    const bool fast_b = uls >= 0x1p-60f && uls <= 0x1p60f;
    const float2 u2_01 = make_float2(2.0f * u0, 2.0f * c01.y), u2_23 = make_float2(2.0f * c23.x, 2.0f * c23.y);
    bool fast_u = fast_b;
    if constexpr (HALF) {
        // Finite binary16 values have |2u| = 0 or within [2^-23, 2^17]; only
        // row `col` (the float ucl - vl) needs the full test.
        const __half2 lim = __float2half2_rn(65504.0f);
        const float m = fabsf(u2_01.x);
        fast_u = fast_u && __hble2(__habs2(t.h[0][0]), lim) && __hble2(__habs2(t.h[0][1]), lim) &&
                 (id != col || m == 0.0f || (m >= 0x1p-32f && m <= 0x1p30f));
    } else {
        const float m[4] = {fabsf(u2_01.x), fabsf(u2_01.y), fabsf(u2_23.x), fabsf(u2_23.y)};
#pragma unroll
        for (int q = 0; q < 4; ++q) fast_u = fast_u && (m[q] == 0.0f || (m[q] >= 0x1p-32f && m[q] <= 0x1p30f));
    }
    const float2 ny = dup2(-y), b2 = dup2(uls);
    if (fast_u && !dots_out) {
        // Every quotient of this thread in range (the common case).  The
        // numerator and the first quotient estimate feed only multiplies and
        // fused multiply-adds, never an add, so the packed multiply cannot be
        // contracted here and rounds each lane as the reference's
        // multiplication does.
#pragma unroll
        for (int i = 0; i < VS; ++i) {
            if (i < VMIN || i < V) {
                const float2 d2 = dup2(sm.out[i]);
                const float2 num01 = mul2(u2_01, d2), num23 = mul2(u2_23, d2);
                const float2 nq01 = mul2(num01, ny), nq23 = mul2(num23, ny);
                const float2 r01 = fma2(nq01, b2, num01), r23 = fma2(nq23, b2, num23);
                const float2 mq01 = fma2(r01, ny, nq01), mq23 = fma2(r23, ny, nq23);   // -RN(num / uls)
                if constexpr (HALF && !NOISE) {
                    // a - q straight from the binary16 a (add.f32.f16); row
                    // id keeps its half when it lies above the column.
                    const __half2 h01 = t.h[i + 1][0], h23 = t.h[i + 1][1];
                    const __half2 n01 = __floats2half2_rn(add_f32_h(__low2half(h01), mq01.x),
                                                          add_f32_h(__high2half(h01), mq01.y));
                    t.h[i][0] = row0 ? n01 : __halves2half2(__low2half(h01), __high2half(n01));
                    t.h[i][1] = __floats2half2_rn(add_f32_h(__low2half(h23), mq23.x),
                                                      add_f32_h(__high2half(h23), mq23.y));
                } else {
                    float2 a01, a23;
                    load_column<HALF, NOISE>(t, i + 1, i + 1, noise, nc, a01, a23);
                    float2 n01 = add2(a01, mq01);
                    const float2 n23 = add2(a23, mq23);
                    if (!row0) n01.x = a01.x;
                    t.set2(i, 0, n01.x, n01.y);
                    t.set2(i, 1, n23.x, n23.y);
                }
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < VS; ++i) {
            if (i < VMIN || i < V) {
                const float dot = sm.out[i];
                const float ad = fabsf(dot);
                const bool fast = fast_u && (ad == 0.0f || (ad >= 0x1p-32f && ad <= 0x1p30f));
                float2 a01, a23;
                load_column<HALF, NOISE>(t, i + 1, i + 1, noise, nc, a01, a23);
                float2 n01, n23;
                if (fast) {
                    const float2 d2 = dup2(dot);
                    const float2 num01 = mul2(u2_01, d2), num23 = mul2(u2_23, d2);
                    const float2 nq01 = mul2(num01, ny), nq23 = mul2(num23, ny);
                    const float2 r01 = fma2(nq01, b2, num01), r23 = fma2(nq23, b2, num23);
                    n01 = add2(a01, fma2(r01, ny, nq01));
                    n23 = add2(a23, fma2(r23, ny, nq23));
                } else {
                    n01 = make_float2(a01.x - div_slow(u2_01.x * dot, uls), a01.y - div_slow(u2_01.y * dot, uls));
                    n23 = make_float2(a23.x - div_slow(u2_23.x * dot, uls), a23.y - div_slow(u2_23.y * dot, uls));
                }
                if (!row0) n01.x = a01.x;
                t.set2(i, 0, n01.x, n01.y);
                t.set2(i, 1, n23.x, n23.y);
            }
        }
    }
}

// The precision form's fit (FP32 QR).  The same Householder reflections in
// float with fused multiply-adds, and one batched reduction per column
// instead of two: because the reflection vector u differs from the column
// itself only in row `col`, every dot product u . a_j equals
// sum_{i>=col} a_col[i] a_j[i] - vl * a_j[col], so the norm and all Gram
// sums of a column are reduced together, and each column's partial sums are
// formed right after the previous column's update.  All packed arithmetic
// pairs rows (q0,q1) and (q2,q3), the tile's register pairs.  It rounds
// differently from the reference and is checked against the fp64 fitter.

// Sum over the CTA of v[0..15] (any order); result k in sm.out[k].  A
// transposing butterfly leaves each lane pair with one value summed over
// the warp; eight warps then meet in shared memory.
template <bool MAX>
__device__ __forceinline__ float op16(float a, float b) {
    return MAX ? fmaxf(a, b) : a + b;
}

// op16<MAX> over the CTA of v[0..15]: sums (MAX = false) or maxima.
template <bool MAX>
__device__ __forceinline__ void block_reduce16(float (&v)[16], FitterSmem& sm) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const bool up = lane & 16;
        const float send = up ? v[k] : v[k + 8], keep = up ? v[k + 8] : v[k];
        v[k] = op16<MAX>(keep, __shfl_xor_sync(kFull, send, 16));
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const bool up = lane & 8;
        const float send = up ? v[k] : v[k + 4], keep = up ? v[k + 4] : v[k];
        v[k] = op16<MAX>(keep, __shfl_xor_sync(kFull, send, 8));
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const bool up = lane & 4;
        const float send = up ? v[k] : v[k + 2], keep = up ? v[k + 2] : v[k];
        v[k] = op16<MAX>(keep, __shfl_xor_sync(kFull, send, 4));
    }
    {
        const bool up = lane & 2;
        const float send = up ? v[0] : v[1], keep = up ? v[1] : v[0];
        v[0] = op16<MAX>(keep, __shfl_xor_sync(kFull, send, 2));
    }
    v[0] = op16<MAX>(v[0], __shfl_xor_sync(kFull, v[0], 1));
    const int idx = ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
    if ((lane & 1) == 0) sm.part[idx * 8 + warp] = v[0];
    __syncthreads();
    if (threadIdx.x < 16) {
        const float* p = sm.part + threadIdx.x * 8;
        sm.out[threadIdx.x] = op16<MAX>(op16<MAX>(op16<MAX>(p[0], p[1]), op16<MAX>(p[2], p[3])),
                                        op16<MAX>(op16<MAX>(p[4], p[5]), op16<MAX>(p[6], p[7])));
    }
    __syncthreads();
}

__device__ __forceinline__ void block_sum16(float (&v)[16], FitterSmem& sm) { block_reduce16<false>(v, sm); }

// Partial sums of column COL, held in tile column COL: v[0] the norm of
// rows >= COL+1, v[1+i] the Gram sum of rows >= COL with column COL+1+i.
// The column loop is unrolled, so every tile index is a constant.
template <int COL>
__device__ __forceinline__ void fast_partials(const Tile<false>& t, int id, FitterSmem& sm, float (&v)[16]) {
    constexpr int V = kBuffers - 1 - COL;
    const float2 c01 = t.p[COL][0], c23 = t.p[COL][1];
    const float2 cn = make_float2(id >= COL + 1 ? c01.x : 0.0f, c01.y);
    const float2 cg = make_float2(id >= COL ? c01.x : 0.0f, c01.y);
    const float2 n = fma2(c23, c23, mul2(cn, cn));
    v[0] = n.x + n.y;
#pragma unroll
    for (int i = 0; i < 15; ++i) {
        if (i < V) {
            const float2 g = fma2(t.p[COL + 1 + i][1], c23, mul2(t.p[COL + 1 + i][0], cg));
            v[1 + i] = g.x + g.y;
        } else {
            v[1 + i] = 0.0f;
        }
    }
    if (id == COL) {   // row COL of every column, for the dot products and u
#pragma unroll
        for (int k = COL; k < kBuffers; ++k) sm.rowc[k - COL] = t.p[k][0].x;
    }
}

template <int COL>
struct FastColumn {
    static __device__ __forceinline__ void run(Tile<false>& t, int id, FitterSmem& sm, float (&v)[16]) {
        constexpr int V = kBuffers - 1 - COL;
        block_sum16(v, sm);
        const float norm2 = sm.out[0];
        const float ucl = sm.rowc[0];
        const float vl = sqrtf(__fmaf_rn(ucl, ucl, norm2));
        const float ucl_new = ucl - vl;
        const float uls = __fmaf_rn(ucl_new, ucl_new, norm2);
        const float2 c01 = t.p[COL][0], c23 = t.p[COL][1];
        if (id < COL) sm.Rm[COL][id] = c01.x;
        if (id == COL) sm.Rm[COL][COL] = vl;
        const bool row0 = id >= COL;
        const float u0 = id == COL ? ucl_new : c01.x;
        const float2 nu01 = make_float2(row0 ? -u0 : 0.0f, -c01.y), nu23 = make_float2(-c23.x, -c23.y);
        const float y2 = 2.0f * __frcp_rn(uls);
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const float dot = __fmaf_rn(-sm.rowc[i + 1], vl, sm.out[i + 1]);   // u . a_j
            const float2 w = dup2(dot * y2);
            t.p[COL + 1 + i][0] = fma2(nu01, w, t.p[COL + 1 + i][0]);
            t.p[COL + 1 + i][1] = fma2(nu23, w, t.p[COL + 1 + i][1]);
        }
        if constexpr (COL + 1 < kFeatures) {
            __syncthreads();   // rowc of this column is read; the next owner may write it
            fast_partials<COL + 1>(t, id, sm, v);
            FastColumn<COL + 1>::run(t, id, sm, v);
        }
    }
};

__device__ __forceinline__ void fit_columns_fast(Tile<false>& t, int id, const float* __restrict__ noise,
                                                 NoiseConst nc, FitterSmem& sm) {
    // The noise of features 1..9 (bmfr.cl:625-627) goes in before the first
    // column's sums; in the reference it enters at the first load and stays.
    const float2 hi = dup2(nc.hi);
#pragma unroll
    for (int k = 1; k < kFeatures; ++k) {
        const float* r = noise + (k - 1) * 4 * kLocal + threadIdx.x;
        t.p[k][0] = fma2(hi, make_float2(r[0], r[kLocal]), t.p[k][0]);
        t.p[k][1] = fma2(hi, make_float2(r[2 * kLocal], r[3 * kLocal]), t.p[k][1]);
    }
    float v[16];
    fast_partials<0>(t, id, sm, v);
    FastColumn<0>::run(t, id, sm, v);
    // The colour columns are tile columns 10..12; move them to 0..2 where
    // the back substitution reads them.
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        t.p[c][0] = t.p[kFeatures + c][0];
        t.p[c][1] = t.p[kFeatures + c][1];
    }
}

// ---------------------------------------------------------------------------
// The precision form's default fit: CholeskyQR2 in FP32.
//
// The ten feature columns A (1024 x 10, scaled, with the noise of features
// 1..9) are factored A = Q R by two Gram passes (CholeskyQR2, Fukaya,
// Nakatsukasa, Yanagisawa and Yamamoto, 2014): R1 = chol(A^T A),
// Q1 = A R1^-1 row by row in registers, R2 = chol(Q1^T Q1), R = R2 R1.  The
// colour columns B ride along in the second pass: Q1^T B is reduced with
// Q1^T Q1, and the Cholesky of that augmented Gram matrix returns
// z = R2^-T Q1^T B = Q^T B, the rows 0..9 of the colour columns that the
// reference's Householder sequence leaves.  The weights are R^-1 z, by two
// triangular solves (R2, then R1).
//
// Each pass is one batched reduction of its Gram entries over the CTA, where
// the Householder sequence reduces once per column; the two Cholesky
// factorisations and the solves run in warp 0 with lane j holding column j.
// The noise of features 1..9 keeps cond(A) below about 1e3, so the first
// pass's FP32 Gram matrix stays positive definite, and the second pass,
// whose matrix is within rounding of the identity, restores the accuracy the
// first one loses: the fitted colours match the fp64 fitter more closely
// than the FP32 Householder sequence does on blocks with fireflies, whose
// large colour norms scale every rounding error of the sequence.  A pivot
// below 2^-20 of its column's squared norm marks the column dependent: its
// row of R and its weight are zero.

constexpr int kGram1 = kFeatures * (kFeatures + 1) / 2;   // 55 entries of A^T A
constexpr int kGram2 = kGram1 + kFeatures * 3;             // + Q1^T B: 85
constexpr int kGramStride = 96;                            // per warp in sm.part
constexpr int kGramChunk = 16;                             // entries reduced per butterfly

// One step of the transposing butterfly over lanes l and l ^ X: each lane
// sends half of its 2H values and keeps the other half summed over the pair.
template <int H, int X, int N>
__device__ __forceinline__ void transpose_step(float (&v)[N], int lane) {
    const bool up = lane & X;
#pragma unroll
    for (int k = 0; k < H; ++k) {
        const float send = up ? v[k] : v[k + H], keep = up ? v[k + H] : v[k];
        v[k] = keep + __shfl_xor_sync(kFull, send, X);
    }
}

// Sum over the warp of C = 16 or 32 values per lane (C - 1 shuffles).  On
// return v[0] holds entry lane (C = 32) or lane >> 1 (C = 16, both lanes of
// a pair hold it).
template <int C>
__device__ __forceinline__ float warp_transpose_sum(float (&v)[C]) {
    const int lane = threadIdx.x & 31;
    if constexpr (C == 32) {
        transpose_step<16, 16>(v, lane);
        transpose_step<8, 8>(v, lane);
        transpose_step<4, 4>(v, lane);
        transpose_step<2, 2>(v, lane);
        transpose_step<1, 1>(v, lane);
    } else {
        transpose_step<8, 16>(v, lane);
        transpose_step<4, 8>(v, lane);
        transpose_step<2, 4>(v, lane);
        transpose_step<1, 2>(v, lane);
        v[0] = v[0] + __shfl_xor_sync(kFull, v[0], 1);
    }
    return v[0];
}

// Sum of a_i * a_j over the thread's four rows.
__device__ __forceinline__ float gram4(const Tile<false>& t, int i, int j) {
    const float2 g = fma2(t.p[i][1], t.p[j][1], mul2(t.p[i][0], t.p[j][0]));
    return g.x + g.y;
}

// Gram entries [BASE, BASE + C): entry tri(i, j) = j(j+1)/2 + i (i <= j) of
// the features' Gram matrix, then (second pass) 55 + 10c + i = column i
// against colour c.  Each warp's sums land in sm.part[warp * 96 + entry].
template <int BASE, int C, bool PASS2>
__device__ __forceinline__ void gram_chunk(const Tile<false>& t, FitterSmem& sm) {
    float v[C];
#pragma unroll
    for (int k = 0; k < C; ++k) v[k] = 0.0f;
#pragma unroll
    for (int j = 0; j < kFeatures; ++j) {
#pragma unroll
        for (int i = 0; i < kFeatures; ++i) {
            const int e = j * (j + 1) / 2 + i;
            if (i <= j && e >= BASE && e < BASE + C) v[e - BASE] = gram4(t, i, j);
        }
    }
    if (PASS2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
#pragma unroll
            for (int i = 0; i < kFeatures; ++i) {
                const int e = kGram1 + kFeatures * c + i;
                if (e >= BASE && e < BASE + C) v[e - BASE] = gram4(t, i, kFeatures + c);
            }
        }
    }
    const float s = warp_transpose_sum<C>(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int e = BASE + (C == 32 ? lane : lane >> 1);
    if ((C == 32 || (lane & 1) == 0) && e < (PASS2 ? kGram2 : kGram1)) sm.part[warp * kGramStride + e] = s;
}

// All Gram entries of a pass in chunks of C.
template <int C, bool PASS2, int BASE = 0>
__device__ __forceinline__ void gram_all(const Tile<false>& t, FitterSmem& sm) {
    gram_chunk<BASE, C, PASS2>(t, sm);
    if constexpr (BASE + C < (PASS2 ? kGram2 : kGram1)) gram_all<C, PASS2, BASE + C>(t, sm);
}

// After the barrier that follows gram_chunk: thread e sums Gram entry e over
// the eight warps into sm.gram (85 threads at once, so warp 0's factorisation
// starts from ten loads per lane instead of eighty).  A barrier follows.
template <bool PASS2>
__device__ __forceinline__ void gram_finish(FitterSmem& sm) {
    const int e = threadIdx.x;
    if (e < (PASS2 ? kGram2 : kGram1)) {
        const float* p = sm.part + e;
        sm.gram[e] = ((p[0] + p[kGramStride]) + (p[2 * kGramStride] + p[3 * kGramStride])) +
                     ((p[4 * kGramStride] + p[5 * kGramStride]) + (p[6 * kGramStride] + p[7 * kGramStride]));
    }
}

// Warp 0, after gram_finish and a barrier: lane j < 10 gathers column j of
// the Gram matrix (g[i], i <= j; zeros below) and stores its diagonal entry
// in diag[j]; lanes 10..12 gather the colour column c = lane - 10 of the
// second pass; other lanes zeros.
template <bool PASS2>
__device__ __forceinline__ void gram_columns(FitterSmem& sm, int lane, float (&g)[kFeatures]) {
#pragma unroll
    for (int i = 0; i < kFeatures; ++i) {
        int e = -1;
        if (lane < kFeatures) e = i <= lane ? lane * (lane + 1) / 2 + i : -1;
        else if (PASS2 && lane < kFeatures + 3) e = kGram1 + kFeatures * (lane - kFeatures) + i;
        const float s = e >= 0 ? sm.gram[e] : 0.0f;
        g[i] = s;
        if (i == lane) sm.diag[i] = s;
    }
    __syncwarp();
}

// Cholesky factorisation by one warp.  In: lane j < 10 holds column j of a
// symmetric matrix (g[i], i <= j), lanes 10..12 right-hand columns, diag[k]
// its diagonal.  Out: lane j holds column j of R (g[i] = R(i, j)), lanes
// 10..12 hold R^-T times their column, and inv[k] = 1 / R(k, k) (0 for a
// dependent column) in shared memory.
// The next pivot, lane k+1's g[k+1] after step k, is formed from that lane's
// own registers and broadcast before the step's other shuffles, so the
// chain of pivots does not wait for them (the same fused multiply-add the
// update below performs in that lane).
__device__ __forceinline__ void chol_lanes(float (&g)[kFeatures], int lane, const float* diag, float* inv) {
    float dnext = __shfl_sync(kFull, g[0], 0);
#pragma unroll
    for (int k = 0; k < kFeatures; ++k) {
        const float d = dnext;
        const bool ok = d > 0x1p-20f * diag[k];
        const float y = ok ? rsqrtf(d) : 0.0f;   // 1 / R(k, k)
        const float r = d * y;
        if (lane == 0) inv[k] = y;
        if (lane == k) g[k] = r;
        else if (lane > k) g[k] = g[k] * y;
        if (k + 1 < kFeatures) dnext = __shfl_sync(kFull, __fmaf_rn(-g[k], g[k], g[k + 1]), k + 1);
#pragma unroll
        for (int i = 0; i < kFeatures; ++i) {
            if (i > k) {
                const float rki = __shfl_sync(kFull, g[k], i);
                if (lane >= i) g[i] = __fmaf_rn(-rki, g[k], g[i]);
            }
        }
    }
    __syncwarp();
}

// The fit of a scaled block (float tile, min/max already applied).
__device__ __forceinline__ void fit_columns_cqr2(Tile<false>& t, const float* __restrict__ noise, NoiseConst nc,
                                                 FitterSmem& sm, float* __restrict__ weights_out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float2 hi = dup2(nc.hi);
#pragma unroll
    for (int k = 1; k < kFeatures; ++k) {   // noise of features 1..9 (bmfr.cl:625-627)
        const float* r = noise + (k - 1) * 4 * kLocal + threadIdx.x;
        t.p[k][0] = fma2(hi, make_float2(r[0], r[kLocal]), t.p[k][0]);
        t.p[k][1] = fma2(hi, make_float2(r[2 * kLocal], r[3 * kLocal]), t.p[k][1]);
    }
    // Pass 1: R1 = chol(A^T A).
    gram_all<kGramChunk, false>(t, sm);
    __syncthreads();
    gram_finish<false>(sm);
    __syncthreads();
    if (warp == 0) {
        float g[kFeatures];
        gram_columns<false>(sm, lane, g);
        chol_lanes(g, lane, sm.diag, sm.inv1);
        if (lane < kFeatures) {
#pragma unroll
            for (int i = 0; i < kFeatures; ++i)
                if (i <= lane) sm.Rm[lane][i] = g[i];
        }
    }
    __syncthreads();
    // Q1 = A R1^-1, one row at a time (forward substitution on row vectors).
#pragma unroll
    for (int j = 0; j < kFeatures; ++j) {
        float2 a0 = t.p[j][0], a1 = t.p[j][1];
#pragma unroll
        for (int i = 0; i < j; ++i) {
            const float2 r = dup2(-sm.Rm[j][i]);
            a0 = fma2(r, t.p[i][0], a0);
            a1 = fma2(r, t.p[i][1], a1);
        }
        const float2 y = dup2(sm.inv1[j]);
        t.p[j][0] = mul2(a0, y);
        t.p[j][1] = mul2(a1, y);
    }
    // Pass 2: R2 = chol(Q1^T Q1) and z = R2^-T Q1^T B.
    gram_all<kGramChunk, true>(t, sm);
    __syncthreads();
    gram_finish<true>(sm);
    __syncthreads();
    if (warp == 0) {
        float g[kFeatures];
        gram_columns<true>(sm, lane, g);
        chol_lanes(g, lane, sm.diag, sm.inv2);
        // R2 v = z in lanes 10..12 (R2(i, j) is lane j's g[i]) ...
        float v[kFeatures];
#pragma unroll
        for (int ii = 0; ii < kFeatures; ++ii) {
            const int i = kFeatures - 1 - ii;
            float s = g[i];
#pragma unroll
            for (int j = i + 1; j < kFeatures; ++j) s = __fmaf_rn(-__shfl_sync(kFull, g[i], j), v[j], s);
            v[i] = s * sm.inv2[i];
        }
        // ... then R1 w = v.
        float w[kFeatures];
#pragma unroll
        for (int ii = 0; ii < kFeatures; ++ii) {
            const int i = kFeatures - 1 - ii;
            float s = v[i];
#pragma unroll
            for (int j = i + 1; j < kFeatures; ++j) s = __fmaf_rn(-sm.Rm[j][i], w[j], s);
            w[i] = s * sm.inv1[i];
        }
        if (lane >= kFeatures && lane < kFeatures + 3) {
#pragma unroll
            for (int k = 0; k < kFeatures; ++k) weights_out[3 * k + (lane - kFeatures)] = w[k];
        }
    }
    __syncthreads();
}

// METHOD: FitMethod; the binary16 tile (HALF) serves kFitReference only.
template <bool HALF, int METHOD = kFitReference>
__device__ __forceinline__ void fit_block(Tile<HALF>& t, const float* __restrict__ noise, NoiseConst nc,
                                          FitterSmem& sm, float* __restrict__ weights_out,
                                          float* __restrict__ mm_out) {
    const int id = work_item_id();
    if constexpr (METHOD != kFitReference && !HALF) {
        // Precision form: the twelve minima and maxima in one transposing
        // butterfly (minima as maxima of the negated values); min and max
        // are exact in any order, so only the sign of a zero bound can
        // differ from the reference's tree.
        float v[16];
#pragma unroll
        for (int f = 0; f < kScaled; ++f) {
            const float2 a01 = t.p[kNotScaled + f][0], a23 = t.p[kNotScaled + f][1];
            v[f] = fmaxf(fmaxf(a01.x, a01.y), fmaxf(a23.x, a23.y));
            v[kScaled + f] = fmaxf(fmaxf(-a01.x, -a01.y), fmaxf(-a23.x, -a23.y));
        }
#pragma unroll
        for (int k = 2 * kScaled; k < 16; ++k) v[k] = -INFINITY;
        block_reduce16<true>(v, sm);
        if (threadIdx.x < 2 * kScaled) {
            const int f = threadIdx.x >> 1;
            mm_out[threadIdx.x] = (threadIdx.x & 1) ? sm.out[f] : -sm.out[kScaled + f];
        }
#pragma unroll
        for (int f = 0; f < kScaled; ++f) {
            const float bmax = sm.out[f], bmin = -sm.out[kScaled + f];
            const float d = bmax - bmin;
            const float2 m = dup2(bmin);
            if constexpr (METHOD == kFitCholQR2) {
                // scale() (bmfr.cl:200-205) by one reciprocal per column.
                const float2 y = dup2(fabsf(d) > 1.0f ? __frcp_rn(d) : 1.0f);
                t.p[kNotScaled + f][0] = mul2(add2(t.p[kNotScaled + f][0], neg2(m)), y);
                t.p[kNotScaled + f][1] = mul2(add2(t.p[kNotScaled + f][1], neg2(m)), y);
            } else {
                const float2 a01 = t.p[kNotScaled + f][0], a23 = t.p[kNotScaled + f][1];
                t.set2(kNotScaled + f, 0, scale_by(a01.x, bmin, bmax), scale_by(a01.y, bmin, bmax));
                t.set2(kNotScaled + f, 1, scale_by(a23.x, bmin, bmax), scale_by(a23.y, bmin, bmax));
            }
        }
        if constexpr (METHOD == kFitCholQR2) {
            fit_columns_cqr2(t, noise, nc, sm, weights_out);
            return;
        } else {
            fit_columns_fast(t, id, noise, nc, sm);
        }
    } else {
        // Min/max scaling of features 4..9 (bmfr.cl:511-542), the
        // reference's reduction tree.
        float mm[12];
#pragma unroll
        for (int f = 0; f < kScaled; ++f) {
            const float2 a01 = t.get2(kNotScaled + f, 0), a23 = t.get2(kNotScaled + f, 1);
            const float a[4] = {a01.x, a01.y, a23.x, a23.y};
            float mx = -INFINITY, mn = INFINITY;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                mx = fmax_cl(a[q], mx);
                mn = fmin_cl(a[q], mn);
            }
            mm[f] = mx;
            mm[kScaled + f] = mn;
        }
        block_reduce<12, 2, 1>(mm, 12, kScaled, sm);
        if (threadIdx.x < 2 * kScaled) {
            const int f = threadIdx.x >> 1;
            mm_out[threadIdx.x] = (threadIdx.x & 1) ? sm.out[f] : sm.out[kScaled + f];
        }
#pragma unroll
        for (int f = 0; f < kScaled; ++f) {
            const float bmax = sm.out[f], bmin = sm.out[kScaled + f];
            const float2 a01 = t.get2(kNotScaled + f, 0), a23 = t.get2(kNotScaled + f, 1);
            t.set2(kNotScaled + f, 0, scale_by(a01.x, bmin, bmax), scale_by(a01.y, bmin, bmax));
            t.set2(kNotScaled + f, 1, scale_by(a23.x, bmin, bmax), scale_by(a23.y, bmin, bmax));
        }
        qr_column<HALF, true>(t, 0, id, noise, nc, sm);
#pragma unroll 1
        for (int col = 1; col < 6; ++col) qr_column<HALF, false, 12, 7>(t, col, id, noise, nc, sm);   // 11..7 later columns
#pragma unroll 1
        for (int col = 6; col < kFeatures; ++col) qr_column<HALF, false, 6, 3>(t, col, id, noise, nc, sm);   // 6..3
    }

    // After ten column steps the colour columns are tile columns 0..2: rows 0..9
    // form R's right-hand side (bmfr.cl:596-600 for col >= 10).
    if (id < kFeatures) {
        sm.rhs[id][0] = t.get2(0, 0).x;
        sm.rhs[id][1] = t.get2(1, 0).x;
        sm.rhs[id][2] = t.get2(2, 0).x;
    }
    __syncthreads();
    // Back substitution (bmfr.cl:659-699): warp c solves colour channel c.
    // Lane x holds column x of R in registers, col[y] = R(x, y) for y <= x;
    // lane 10 holds the right-hand side; the other lanes hold zeros.  Each
    // step of the reference's work-group loop becomes shuffles within the warp.
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp < 3) {
        const int c = warp;
        float col[kFeatures];
#pragma unroll
        for (int y = 0; y < kFeatures; ++y) {
            float v = 0.0f;
            if (lane < kFeatures && y <= lane) v = sm.Rm[lane][y];
            if (lane == kFeatures) v = sm.rhs[y][c];
            col[y] = v;
        }
#pragma unroll
        for (int i = kREdge - 2; i >= 0; --i) {
            const float dv = __shfl_sync(kFull, col[i], i);               // R(i, i)
            if (lane >= i && lane < kREdge) col[i] = col[i] / dv;        // R(x, i) /= R(i, i), x = i..10
            float sub[kFeatures];
#pragma unroll
            for (int j = i + 1; j < kREdge - 1; ++j) sub[j] = __shfl_sync(kFull, col[i], j);
            if (lane == kREdge - 1) {                                    // R(10, i) -= R(j, i), j = i+1..9
                float v = col[i];
#pragma unroll
                for (int j = i + 1; j < kREdge - 1; ++j) v = v - sub[j];
                col[i] = v;
            }
            const float xi = __shfl_sync(kFull, col[i], kREdge - 1);      // R(10, i), solved
            if (lane == i) {                                             // R(i, y) *= R(10, i), y <= i
#pragma unroll
                for (int y = 0; y <= i; ++y) col[y] = col[y] * xi;
            }
        }
        if (lane == kREdge - 1) {
#pragma unroll
            for (int k = 0; k < kFeatures; ++k) weights_out[3 * k + c] = col[k];
        }
    }
    __syncthreads();
}

}  // namespace bmfr
