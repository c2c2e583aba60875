// scene_gpu.cu — the procedural G-buffer source rendered on the device, so
// that many-stream workloads do not wait on the host renderer or on uploads.
// Same scene, camera and noise model as scene.cpp (shared through
// scene_internal.h); the arithmetic is float and the noise uniforms come
// from the same 64-bit counter hash, so images match the host renderer's to
// float rounding rather than bit for bit.
#include <cuda_runtime.h>

#include "bmfr_scene.h"
#include "scene_internal.h"

namespace {

constexpr int kMaxSpheres = 64;

struct DevSphere {
    float cx, cy, cz, r;
    float albedo[3];
};

struct DevScene {
    DevSphere spheres[kMaxSpheres];
    int sphere_count;
    float plane_albedo[3];
    float eye[3], right[3], up[3], fwd[3];
    float tan_half, aspect, ext;
    float light[3];
    float noise_mu, noise_sigma, firefly_fraction, firefly_scale;
    unsigned long long seed;
    int frame, width, height;
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long& s) {
    unsigned long long z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Uniform in (0,1) from (seed, frame, pixel, lane), as the host's hash_u01.
__device__ __forceinline__ float hash_u01f(unsigned long long seed, unsigned long long frame,
                                           unsigned long long pixel, unsigned long long lane) {
    unsigned long long s = seed ^ (frame * 0xd1b54a32d192ed03ull) ^ (pixel * 0xabc98388fb8fac03ull) ^
                           (lane * 0x8cb92ba72f3d8dd7ull);
    mix64(s);
    return ((float)(mix64(s) >> 40) + 0.5f) * (1.0f / 16777216.0f);
}

__global__ void k_render(DevScene sc, float* __restrict__ albedo, float* __restrict__ normals,
                         float* __restrict__ positions, float* __restrict__ noisy, float* __restrict__ clean) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= sc.width || y >= sc.height) return;
    const size_t i = (size_t)y * sc.width + x;
    const float nx = ((x + 0.5f) / sc.width) * 2.0f - 1.0f;
    const float ny = ((y + 0.5f) / sc.height) * 2.0f - 1.0f;
    const float a = nx * sc.aspect * sc.tan_half, bq = -ny * sc.tan_half;
    float dx = sc.right[0] * a + sc.up[0] * bq + sc.fwd[0];
    float dy = sc.right[1] * a + sc.up[1] * bq + sc.fwd[1];
    float dz = sc.right[2] * a + sc.up[2] * bq + sc.fwd[2];
    const float inv = rsqrtf(dx * dx + dy * dy + dz * dz);
    dx *= inv;
    dy *= inv;
    dz *= inv;
    float best = 1e30f;
    int hit = -2;
    if (dy < 0.0f) {
        const float t = -sc.eye[1] / dy;
        const float px = sc.eye[0] + dx * t, pz = sc.eye[2] + dz * t;
        if (t > 1e-4f && fabsf(px) <= sc.ext && fabsf(pz) <= sc.ext) {
            best = t;
            hit = -1;
        }
    }
    for (int k = 0; k < sc.sphere_count; ++k) {
        const DevSphere& sp = sc.spheres[k];
        const float ox = sc.eye[0] - sp.cx, oy = sc.eye[1] - sp.cy, oz = sc.eye[2] - sp.cz;
        const float b = ox * dx + oy * dy + oz * dz;
        const float c = ox * ox + oy * oy + oz * oz - sp.r * sp.r;
        const float disc = b * b - c;
        if (disc < 0.0f) continue;
        const float sq = sqrtf(disc);
        float t = -b - sq;
        if (t <= 1e-4f) t = -b + sq;
        if (t > 1e-4f && t < best) {
            best = t;
            hit = k;
        }
    }
    float* P = positions + 3 * i;
    float* N = normals + 3 * i;
    float* A = albedo + 3 * i;
    float* C = noisy + 3 * i;
    if (hit == -2) {
        for (int c = 0; c < 3; ++c) P[c] = N[c] = A[c] = C[c] = 0.0f;
        if (clean)
            for (int c = 0; c < 3; ++c) clean[3 * i + c] = 0.0f;
        return;
    }
    float p[3] = {sc.eye[0] + dx * best, sc.eye[1] + dy * best, sc.eye[2] + dz * best};
    float n[3];
    const float* alb;
    if (hit == -1) {
        p[1] = 0.0f;
        n[0] = 0.0f;
        n[1] = 1.0f;
        n[2] = 0.0f;
        alb = sc.plane_albedo;
    } else {
        const DevSphere& sp = sc.spheres[hit];
        n[0] = p[0] - sp.cx;
        n[1] = p[1] - sp.cy;
        n[2] = p[2] - sp.cz;
        const float l = rsqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        n[0] *= l;
        n[1] *= l;
        n[2] *= l;
        alb = sp.albedo;
    }
    for (int c = 0; c < 3; ++c) {
        P[c] = p[c] + 0.0f;   // no negative zero
        N[c] = n[c] + 0.0f;
    }
    const float shade = fmaxf(0.0f, n[0] * sc.light[0] + n[1] * sc.light[1] + n[2] * sc.light[2]) + 0.1f;
    const bool firefly = hash_u01f(sc.seed, sc.frame, i, 7) < sc.firefly_fraction;
    for (int c = 0; c < 3; ++c) {
        A[c] = alb[c];
        const float u1 = hash_u01f(sc.seed, sc.frame, i, 2 * c);
        const float u2 = hash_u01f(sc.seed, sc.frame, i, 2 * c + 1);
        const float g = sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
        float xv = expf(sc.noise_mu + sc.noise_sigma * g);
        if (firefly) xv *= sc.firefly_scale;
        C[c] = shade * xv;
        if (clean) clean[3 * i + c] = fminf(1.0f, powf(fmaxf(0.0f, alb[c] * shade), 0.454545f));
    }
}

}  // namespace

extern "C" int bmfr_scene_render_device(const bmfr_scene_desc* d, int frame, float* albedo, float* normals,
                                        float* positions, float* noisy, float* clean, void* stream) {
    using namespace bmfr_scene_internal;
    if (!d || !albedo || !normals || !positions || !noisy || frame < 0) return -1;
    if (d->sphere_count > kMaxSpheres) return -1;
    const Scene s = build_scene(d);
    const Camera cam = make_camera(d, frame);
    DevScene sc;
    for (int k = 0; k < d->sphere_count; ++k) {
        const Sphere& sp = s.spheres[k];
        sc.spheres[k] = DevSphere{(float)sp.c.x, (float)sp.c.y, (float)sp.c.z, (float)sp.r,
                                  {sp.albedo[0], sp.albedo[1], sp.albedo[2]}};
    }
    sc.sphere_count = d->sphere_count;
    for (int c = 0; c < 3; ++c) sc.plane_albedo[c] = s.plane_albedo[c];
    const V3 v3[4] = {cam.eye, cam.right, cam.up, cam.fwd};
    float* dst[4] = {sc.eye, sc.right, sc.up, sc.fwd};
    for (int k = 0; k < 4; ++k) {
        dst[k][0] = (float)v3[k].x;
        dst[k][1] = (float)v3[k].y;
        dst[k][2] = (float)v3[k].z;
    }
    sc.tan_half = (float)cam.tan_half;
    sc.aspect = (float)cam.aspect;
    sc.ext = d->plane_half_extent;
    const V3 light = normalize(V3{0.4, 1.0, 0.3});
    sc.light[0] = (float)light.x;
    sc.light[1] = (float)light.y;
    sc.light[2] = (float)light.z;
    sc.noise_mu = d->noise_mu;
    sc.noise_sigma = d->noise_sigma;
    sc.firefly_fraction = d->firefly_fraction;
    sc.firefly_scale = d->firefly_scale;
    sc.seed = d->seed;
    sc.frame = frame;
    sc.width = d->width;
    sc.height = d->height;
    const dim3 block(32, 8), grid((d->width + 31) / 32, (d->height + 7) / 8);
    k_render<<<grid, block, 0, (cudaStream_t)stream>>>(sc, albedo, normals, positions, noisy, clean);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
