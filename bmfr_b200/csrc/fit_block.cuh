// fit_block.cuh — the per-block least-squares fit of BMFR (opencl/bmfr.cl:
// 490-700) as a device routine for one 256-thread CTA, shared by the
// standalone fitter kernel and the fused accumulate+fit kernel.
//
// Layout.  Each thread is one of the reference's 256 work-items and owns the
// same four pixels of the 32x32 block (rows id, id+256, id+512, id+768 of the
// 1024x13 matrix).  The whole block stays in registers, t[13][4], through the
// min/max scaling, the ten Householder reflections and their updates; tmp
// data is never written back.  Work-item ids are assigned to lanes as
//     id = 8*warp + (lane & 7) + 64*(lane >> 3)
// so that the first stage of the reference's reduction tree (ids i, i+64,
// i+128, i+192, bmfr.cl:32-33) sits inside one warp and runs on shuffles.
//
// Reductions.  block_reduce evaluates parallel_reduction_sum/min/max
// (bmfr.cl:25-87) over exactly the same tree, so the sums round exactly as
// the reference's do, and batches V independent reductions behind one pair of
// barriers: the twelve min/max values of the scaling step, and per column the
// up to twelve dot products, which are independent once the Householder
// vector is known.  A column costs two batched reductions (norm, dots) — four
// barriers — where the reference spends three barriers per dot product.
//
// The colour columns' own reflections (columns 10..12, bmfr.cl:549 with
// col_limited = 10) only change rows >= 10, which neither the back
// substitution nor the weights read (bmfr.cl:660-699), so they are skipped.
#pragma once

#include "common.cuh"

namespace bmfr {

struct FitterSmem {
    float part[12 * 64];   // first-stage partial sums, 64 per batched value
    float out[12];         // reduction results
    float ucl;             // u[col] broadcast from its owner
    float Rm[10][10];      // R of the ten feature columns: Rm[x][y], y <= x
    float rhs[10][3];      // rows 0..9 of the three colour columns
    float Rb[3][11][11];   // per-channel copy used by the back substitution
};

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int work_item_id() {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    return 8 * warp + (lane & 7) + 64 * (lane >> 3);
}

// OP: 0 sum, 1 min, 2 max.  Values [0, SPLIT) use OP_A, [SPLIT, V) use OP_B.
template <int OP>
__device__ __forceinline__ float rop(float a, float b) {
    if (OP == 0) return a + b;
    if (OP == 1) return fmin_cl(a, b);
    return fmax_cl(a, b);
}

template <int V, int SPLIT, int OP_A, int OP_B>
__device__ __forceinline__ void block_reduce(const float (&v)[V], FitterSmem& sm) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < V; ++i) {
        const float a = v[i];
        const float b = __shfl_down_sync(kFull, a, 8);
        const float c = __shfl_down_sync(kFull, a, 16);
        const float d = __shfl_down_sync(kFull, a, 24);
        float s1;
        if (i < SPLIT) {
            if (OP_A == 0) s1 = a + ((b + c) + d);          // bmfr.cl:33
            else s1 = rop<OP_A>(rop<OP_A>(rop<OP_A>(a, b), c), d);   // bmfr.cl:52-53, 74-75
        } else {
            if (OP_B == 0) s1 = a + ((b + c) + d);
            else s1 = rop<OP_B>(rop<OP_B>(rop<OP_B>(a, b), c), d);
        }
        if (lane < 8) sm.part[i * 64 + 8 * warp + lane] = s1;
    }
    __syncthreads();
    // Stages 2 and 3: value vi is finished by the 8-lane group `lane >> 3` of
    // warp vi % 8; lane j of the group forms sum_vec[j] (bmfr.cl:35-37).
    const int vi = warp + 8 * (lane >> 3);
    const int j = lane & 7;
    float s2 = 0.0f;
    const bool first = vi < SPLIT;
    if (vi < V) {
        const float* p = sm.part + vi * 64 + j;
        const int op = first ? OP_A : OP_B;
        if (op == 0) {
            float acc = p[8];
#pragma unroll
            for (int m = 2; m < 8; ++m) acc = acc + p[8 * m];
            s2 = p[0] + acc;
        } else if (op == 1) {
            float acc = p[0];
#pragma unroll
            for (int m = 1; m < 8; ++m) acc = fmin_cl(acc, p[8 * m]);
            s2 = acc;
        } else {
            float acc = p[0];
#pragma unroll
            for (int m = 1; m < 8; ++m) acc = fmax_cl(acc, p[8 * m]);
            s2 = acc;
        }
    }
    // Stage 3 (bmfr.cl:39-42): sum_vec[0] + ... + sum_vec[7], left to right.
    const int base = lane & ~7;
    float r = __shfl_sync(kFull, s2, base);
#pragma unroll
    for (int m = 1; m < 8; ++m) {
        const float x = __shfl_sync(kFull, s2, base + m);
        const int op = first ? OP_A : OP_B;
        r = op == 0 ? r + x : (op == 1 ? fmin_cl(r, x) : fmax_cl(r, x));
    }
    if (vi < V && j == 0) sm.out[vi] = r;
    __syncthreads();
}

template <bool ROUND>
__device__ __forceinline__ float stq(float v) {
    return ROUND ? round_half(v) : v;
}

// One Householder column (bmfr.cl:549-655) for COL < 10, then the next.
template <int COL, bool ROUND>
struct QrColumn {
    static __device__ __forceinline__ void run(float (&t)[kBuffers][4], int id, int frame, NoiseConst nc,
                                               FitterSmem& sm) {
        // Norm of rows >= COL+1 (bmfr.cl:553-569).
        float nv[1];
        {
            float s = 0.0f;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (id + kLocal * q >= COL + 1) s = s + t[COL][q] * t[COL][q];
            nv[0] = s;
        }
        if (id == COL) sm.ucl = t[COL][0];
        block_reduce<1, 1, 0, 0>(nv, sm);
        const float norm2 = sm.out[0];
        const float ucl = sm.ucl;
        // Work-item COL's step (bmfr.cl:580-588), evaluated by everyone.
        const float vl = sqrtf(norm2 + ucl * ucl);
        const float ucl_new = ucl - vl;
        const float uls = norm2 + ucl_new * ucl_new;
        if (id < COL) sm.Rm[COL][id] = t[COL][0];
        if (id == COL) sm.Rm[COL][COL] = vl;
        float u[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) u[q] = t[COL][q];
        if (id == COL) u[0] = ucl_new;

        if (COL == 0) {   // noise on the first load of features 1..9 (bmfr.cl:625-627)
#pragma unroll
            for (int fb = 1; fb < kFeatures; ++fb)
#pragma unroll
                for (int q = 0; q < 4; ++q) t[fb][q] = add_noise(t[fb][q], noise_index(id, q, fb, frame), nc);
        }
        // Dot products with every later column (bmfr.cl:606-638).
        constexpr int V = kBuffers - 1 - COL;
        float d[V];
#pragma unroll
        for (int i = 0; i < V; ++i) {
            float s = 0.0f;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (id + kLocal * q >= COL) s = s + t[COL + 1 + i][q] * u[q];
            d[i] = s;
        }
        block_reduce<V, V, 0, 0>(d, sm);
        // Rank-one update, rounded at the reference's store (bmfr.cl:640-652).
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const float dot = sm.out[i];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (id + kLocal * q >= COL)
                    t[COL + 1 + i][q] = stq<ROUND>(t[COL + 1 + i][q] - ((2.0f * u[q]) * dot) / uls);
        }
        QrColumn<COL + 1, ROUND>::run(t, id, frame, nc, sm);
    }
};
template <bool ROUND>
struct QrColumn<kFeatures, ROUND> {
    static __device__ __forceinline__ void run(float (&)[kBuffers][4], int, int, NoiseConst, FitterSmem&) {}
};

// Fits one block held in t (the values as loaded from tmp_data) and writes
// its 30 weights and 12 min/max values.
template <bool ROUND>
__device__ __forceinline__ void fit_block(float (&t)[kBuffers][4], int frame, NoiseConst nc, FitterSmem& sm,
                                          float* __restrict__ weights_out, float* __restrict__ mm_out) {
    const int id = work_item_id();
    // Min/max scaling of features 4..9 (bmfr.cl:511-542).
    float mm[12];
#pragma unroll
    for (int f = 0; f < kScaled; ++f) {
        float mx = -INFINITY, mn = INFINITY;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            mx = fmax_cl(t[kNotScaled + f][q], mx);
            mn = fmin_cl(t[kNotScaled + f][q], mn);
        }
        mm[f] = mx;
        mm[kScaled + f] = mn;
    }
    block_reduce<12, kScaled, 2, 1>(mm, sm);
    if (threadIdx.x < 2 * kScaled) {
        const int f = threadIdx.x >> 1;
        mm_out[threadIdx.x] = (threadIdx.x & 1) ? sm.out[f] : sm.out[kScaled + f];
    }
#pragma unroll
    for (int f = 0; f < kScaled; ++f) {
        const float bmax = sm.out[f], bmin = sm.out[kScaled + f];
#pragma unroll
        for (int q = 0; q < 4; ++q) t[kNotScaled + f][q] = stq<ROUND>(scale(t[kNotScaled + f][q], bmin, bmax));
    }

    QrColumn<0, ROUND>::run(t, id, frame, nc, sm);

    // R of the colour columns, rows 0..9 (bmfr.cl:596-600 for col >= 10).
    if (id < kFeatures) {
        sm.rhs[id][0] = t[kFeatures][0];
        sm.rhs[id][1] = t[kFeatures + 1][0];
        sm.rhs[id][2] = t[kFeatures + 2][0];
    }
    __syncthreads();
    // Back substitution, one thread per colour channel (bmfr.cl:659-699).
    if (threadIdx.x < 3) {
        const int c = threadIdx.x;
        float(*R)[kREdge] = sm.Rb[c];
        for (int x = 0; x < kFeatures; ++x)
            for (int y = 0; y <= x; ++y) R[x][y] = sm.Rm[x][y];
        for (int y = 0; y < kFeatures; ++y) R[kFeatures][y] = sm.rhs[y][c];
        for (int i = kREdge - 2; i >= 0; --i) {
            const float dv = R[i][i];
            for (int x = i; x < kREdge; ++x) R[x][i] = R[x][i] / dv;
            for (int j = i + 1; j < kREdge - 1; ++j) R[kREdge - 1][i] = R[kREdge - 1][i] - R[j][i];
            for (int y = 0; y <= i; ++y) R[i][y] = R[i][y] * R[kREdge - 1][i];
        }
        for (int k = 0; k < kFeatures; ++k) weights_out[3 * k + c] = R[kREdge - 1][k];
    }
}

}  // namespace bmfr
