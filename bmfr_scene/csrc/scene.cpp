// scene.cpp — seeded procedural G-buffer renderer (host cores, OpenMP).
// Stands in for the reference's EXR dataset and camera_matrices.h
// (opencl/bmfr.cpp:44-53, 145-172, 252-307); see include/bmfr_scene.h.
#include "bmfr_scene.h"
#include "scene_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif



namespace {
using namespace bmfr_scene_internal;

inline float canon(double v) { return (float)v + 0.0f; }   // no negative zero

}  // namespace

extern "C" {

int bmfr_scene_default(bmfr_scene_desc* d, uint64_t seed, int width, int height,
                       int sphere_count) {
    if (!d || width <= 0 || height <= 0 || sphere_count < 0) return -1;
    std::memset(d, 0, sizeof *d);
    d->seed = seed;
    d->width = width;
    d->height = height;
    d->sphere_count = sphere_count;
    d->orbit_degrees_per_frame = 0.5f;
    d->orbit_start_degrees = 30.0f;
    d->orbit_radius = 10.0f;
    d->camera_height = 3.0f;
    d->vertical_fov_degrees = 60.0f;
    d->noise_mu = -0.5f;
    d->noise_sigma = 1.0f;
    d->firefly_fraction = 0.001f;
    d->firefly_scale = 100.0f;
    d->plane_half_extent = 64.0f;
    d->position_limit_squared = 0.01f;
    d->normal_limit_squared = 0.1f;
    return 0;
}

int bmfr_scene_camera(const bmfr_scene_desc* d, int frame, float m[16]) {
    if (!d || !m || frame < 0) return -1;
    const Camera cam = make_camera(d, frame);
    // camera_matrices[f][i][j] = VP[j][i]: clip = p^T M (bmfr.cl:343-347).
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) m[i * 4 + j] = (float)cam.vp[j][i];
    return 0;
}

int bmfr_scene_pixel_offset(const bmfr_scene_desc* d, int frame, float off[2]) {
    if (!d || !off || frame < 0) return -1;
    off[0] = 0.5f;
    off[1] = 0.5f;
    return 0;
}

int bmfr_scene_render(const bmfr_scene_desc* d, int frame, float* albedo, float* normals,
                      float* positions, float* noisy, float* clean, int threads) {
    if (!d || !albedo || !normals || !positions || !noisy || frame < 0) return -1;
    const Scene sc = build_scene(d);
    const Camera cam = make_camera(d, frame);
    const V3 light = normalize(V3{0.4, 1.0, 0.3});
    const int W = d->width, H = d->height;
    const double ext = d->plane_half_extent;
#ifdef _OPENMP
    const int nt = threads > 0 ? threads : omp_get_max_threads();
#else
    (void)threads;
#endif
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const size_t i = (size_t)y * W + x;
            const double nx = ((x + 0.5) / W) * 2.0 - 1.0;
            const double ny = ((y + 0.5) / H) * 2.0 - 1.0;
            // Inverse of the flipped projection: camera-space direction.
            const V3 dir = normalize(cam.right * (nx * cam.aspect * cam.tan_half) +
                                     cam.up * (-ny * cam.tan_half) + cam.fwd);
            double best = 1e30;
            int hit = -2;   // -2 miss, -1 plane, >=0 sphere
            if (dir.y < 0.0) {
                const double t = -cam.eye.y / dir.y;
                const V3 p = cam.eye + dir * t;
                if (t > 1e-4 && std::fabs(p.x) <= ext && std::fabs(p.z) <= ext) {
                    best = t;
                    hit = -1;
                }
            }
            for (size_t k = 0; k < sc.spheres.size(); ++k) {
                const Sphere& sp = sc.spheres[k];
                const V3 oc = cam.eye - sp.c;
                const double b = dot(oc, dir);
                const double c = dot(oc, oc) - sp.r * sp.r;
                const double disc = b * b - c;
                if (disc < 0.0) continue;
                const double sq = std::sqrt(disc);
                double t = -b - sq;
                if (t <= 1e-4) t = -b + sq;
                if (t > 1e-4 && t < best) {
                    best = t;
                    hit = (int)k;
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
                continue;
            }
            V3 p = cam.eye + dir * best;
            V3 n;
            const float* alb;
            if (hit == -1) {
                p.y = 0.0;
                n = {0.0, 1.0, 0.0};
                alb = sc.plane_albedo;
            } else {
                n = normalize(p - sc.spheres[hit].c);
                alb = sc.spheres[hit].albedo;
            }
            P[0] = canon(p.x);
            P[1] = canon(p.y);
            P[2] = canon(p.z);
            N[0] = canon(n.x);
            N[1] = canon(n.y);
            N[2] = canon(n.z);
            const double shade = std::max(0.0, dot(n, light)) + 0.1;
            const bool firefly = hash_u01(d->seed, frame, i, 7) < d->firefly_fraction;
            for (int c = 0; c < 3; ++c) {
                A[c] = alb[c];
                const double u1 = hash_u01(d->seed, frame, i, 2 * c);
                const double u2 = hash_u01(d->seed, frame, i, 2 * c + 1);
                const double g = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
                double xval = std::exp(d->noise_mu + d->noise_sigma * g);
                if (firefly) xval *= d->firefly_scale;
                C[c] = (float)(shade * xval);
                if (clean) {
                    const double v = std::max(0.0, (double)alb[c] * shade);
                    clean[3 * i + c] = (float)std::min(1.0, std::pow(v, 0.454545));
                }
            }
        }
    }
    return 0;
}

}  // extern "C"
