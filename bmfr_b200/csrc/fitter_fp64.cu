// fitter_fp64.cu — the fitter in double precision (the precision form's
// reference, and the only FP64 code on the device).
//
// It restates opencl/bmfr.cl:490-700 with every value in double and no
// intermediate rounding: the min/max scaling of features 4..9, the ten
// Householder reflections over the same reduction tree as
// parallel_reduction_sum (bmfr.cl:25-44), the feature noise formed in double
// as the reference's double literal NOISE_AMOUNT does, and the back
// substitution.  One 256-thread CTA per block keeps the 1024x13 block in
// shared memory (104 KB); speed is not its purpose.
#include "common.cuh"
#include "kernels.h"

namespace bmfr {

namespace {

struct Fp64Smem {
    double tile[kBuffers][kBlockPixels];
    double u[kBlockPixels];
    double sv[kLocal];
    double R[kREdge][kREdge][3];
    double red;
    float mn, mx;
};

// parallel_reduction_sum (bmfr.cl:26-44) over sv[0..255]; every thread gets the sum.
__device__ double reduce_sum_d(Fp64Smem& S) {
    const int id = threadIdx.x;
    __syncthreads();
    if (id < 64) S.sv[id] = S.sv[id] + ((S.sv[id + 64] + S.sv[id + 128]) + S.sv[id + 192]);
    __syncthreads();
    if (id < 8) {
        double acc = S.sv[id + 8];
        for (int m = 2; m < 8; ++m) acc = acc + S.sv[id + 8 * m];
        S.sv[id] = S.sv[id] + acc;
    }
    __syncthreads();
    if (id == 0) {
        double r = S.sv[0];
        for (int m = 1; m < 8; ++m) r = r + S.sv[m];
        S.red = r;
    }
    __syncthreads();
    return S.red;
}

}  // namespace

__global__ void __launch_bounds__(256) k_fitter_fp64(int frame, double noise2, const void* __restrict__ tmp,
                                                     int half_tmp, double* __restrict__ weights,
                                                     float* __restrict__ mins_maxs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Fp64Smem& S = *reinterpret_cast<Fp64Smem*>(smem_raw);
    const int b = blockIdx.x, id = threadIdx.x;
    const size_t base = (size_t)b * kBuffers * kBlockPixels;
    for (int i = id; i < kBuffers * kBlockPixels; i += kLocal) {
        const double v = half_tmp ? (double)__half2float(reinterpret_cast<const __half*>(tmp)[base + i])
                                  : (double)reinterpret_cast<const float*>(tmp)[base + i];
        S.tile[i / kBlockPixels][i % kBlockPixels] = v;
    }
    __syncthreads();
    // Scaling (bmfr.cl:511-542); min and max are exact in any order.
    for (int fb = kNotScaled; fb < kBuffers - 3; ++fb) {
        if (id == 0) {
            float mn = INFINITY, mx = -INFINITY;
            for (int i = 0; i < kBlockPixels; ++i) {
                const float v = (float)S.tile[fb][i];
                mn = fmin_cl(v, mn);
                mx = fmax_cl(v, mx);
            }
            S.mn = mn;
            S.mx = mx;
            mins_maxs[((size_t)b * kScaled + fb - kNotScaled) * 2 + 0] = mn;
            mins_maxs[((size_t)b * kScaled + fb - kNotScaled) * 2 + 1] = mx;
        }
        __syncthreads();
        const double mn = S.mn, mx = S.mx;
        for (int i = id; i < kBlockPixels; i += kLocal) {
            const double v = S.tile[fb][i];
            S.tile[fb][i] = fabs(mx - mn) > 1.0 ? (v - mn) / (mx - mn) : v - mn;
        }
        __syncthreads();
    }
    // Householder columns 0..9 (bmfr.cl:549-655).
    for (int col = 0; col < kFeatures; ++col) {
        double s = 0.0;
        for (int q = 0; q < 4; ++q) {
            const int idx = id + kLocal * q;
            const double a = S.tile[col][idx];
            S.u[idx] = a;
            if (idx >= col + 1) s = s + a * a;
        }
        S.sv[id] = s;
        const double norm2 = reduce_sum_d(S);
        const double ucl = S.u[col];
        const double vl = sqrt(norm2 + ucl * ucl);
        const double ucl_new = ucl - vl;
        const double uls = norm2 + ucl_new * ucl_new;
        if (id <= kREdge - 1) {
            const double r = id < col ? S.u[id] : (id == col ? vl : 0.0);
            for (int c = 0; c < 3; ++c) S.R[col][id][c] = r;
        }
        __syncthreads();
        if (id == 0) S.u[col] = ucl_new;
        __syncthreads();
        for (int fb = col + 1; fb < kBuffers; ++fb) {
            double acc = 0.0;
            double cache[4];
            for (int q = 0; q < 4; ++q) {
                const int idx = id + kLocal * q;
                if (idx >= col) {
                    double v = S.tile[fb][idx];
                    if (col == 0 && fb < kFeatures) {
                        const float r = hash_random(noise_index(id, q, fb, frame)) - 0.5f;
                        v = v + noise2 * (double)r;
                    }
                    cache[q] = v;
                    acc = acc + v * S.u[idx];
                }
            }
            S.sv[id] = acc;
            const double dot = reduce_sum_d(S);
            for (int q = 0; q < 4; ++q) {
                const int idx = id + kLocal * q;
                if (idx >= col) S.tile[fb][idx] = cache[q] - ((2.0 * S.u[idx]) * dot) / uls;
            }
            __syncthreads();
        }
    }
    // Back substitution (bmfr.cl:659-699) on rows 0..9 of the colour columns.
    if (id < 3) {
        const int c = id;
        for (int y = 0; y < kFeatures; ++y) S.R[kREdge - 1][y][c] = S.tile[kFeatures + c][y];
        for (int i = kREdge - 2; i >= 0; --i) {
            const double dv = S.R[i][i][c];
            for (int x = i; x < kREdge; ++x) S.R[x][i][c] = S.R[x][i][c] / dv;
            for (int j = i + 1; j < kREdge - 1; ++j) S.R[kREdge - 1][i][c] = S.R[kREdge - 1][i][c] - S.R[j][i][c];
            for (int y = 0; y <= i; ++y) S.R[i][y][c] = S.R[i][y][c] * S.R[kREdge - 1][i][c];
        }
        for (int k = 0; k < kFeatures; ++k) weights[((size_t)b * kFeatures + k) * 3 + c] = S.R[kREdge - 1][k][c];
    }
}

cudaError_t launch_fitter_fp64(const Geometry& g, int frame, double noise_amount, const void* tmp, bool half_tmp,
                               double* weights, float* mins_maxs, cudaStream_t s) {
    const int smem = (int)sizeof(Fp64Smem);
    cudaError_t e = cudaFuncSetAttribute(k_fitter_fp64, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    k_fitter_fp64<<<g.blocks, kLocal, smem, s>>>(frame, noise_amount * 2.0, tmp, half_tmp ? 1 : 0, weights,
                                                  mins_maxs);
    return cudaGetLastError();
}

}  // namespace bmfr
