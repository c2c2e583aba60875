// scene_internal.h — procedural scene and camera shared by the host renderer
// (scene.cpp) and the device renderer (scene_gpu.cu).  Internal.
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

#include "bmfr_scene.h"

namespace bmfr_scene_internal {
struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V3 normalize(V3 a) { return a * (1.0 / std::sqrt(dot(a, a))); }

inline uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
inline double u01(uint64_t& s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

// Counter-based uniform in (0,1) from (seed, frame, pixel, lane).
inline double hash_u01(uint64_t seed, uint64_t frame, uint64_t pixel, uint64_t lane) {
    uint64_t s = seed ^ (frame * 0xd1b54a32d192ed03ull) ^ (pixel * 0xabc98388fb8fac03ull) ^
                 (lane * 0x8cb92ba72f3d8dd7ull);
    splitmix64(s);
    return ((double)(splitmix64(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

struct Sphere {
    V3 c;
    double r;
    float albedo[3];
};

struct Scene {
    std::vector<Sphere> spheres;
    float plane_albedo[3];
};

inline Scene build_scene(const bmfr_scene_desc* d) {
    Scene sc;
    uint64_t s = d->seed * 0x2545f4914f6cdd1dull + 0x1234567ull;
    for (int c = 0; c < 3; ++c) sc.plane_albedo[c] = (float)(0.05 + 0.9 * u01(s));
    for (int i = 0; i < d->sphere_count; ++i) {
        Sphere sp;
        sp.r = 0.3 + 1.2 * u01(s);
        const double cx = -5.0 + 10.0 * u01(s);
        const double cz = -5.0 + 10.0 * u01(s);
        sp.c = {cx, sp.r, cz};   // resting on the plane
        for (int c = 0; c < 3; ++c) sp.albedo[c] = (float)(0.05 + 0.9 * u01(s));
        sc.spheres.push_back(sp);
    }
    return sc;
}

struct Camera {
    V3 eye, right, up, fwd;
    double tan_half, aspect;
    double vp[4][4];   // column-vector view-projection
};

inline Camera make_camera(const bmfr_scene_desc* d, int frame) {
    Camera cam;
    const double deg = d->orbit_start_degrees + (double)frame * d->orbit_degrees_per_frame;
    const double th = deg * M_PI / 180.0;
    cam.eye = {d->orbit_radius * std::cos(th), d->camera_height, d->orbit_radius * std::sin(th)};
    const V3 target = {0.0, 0.5, 0.0};
    cam.fwd = normalize(target - cam.eye);
    cam.right = normalize(cross(cam.fwd, V3{0.0, 1.0, 0.0}));
    cam.up = cross(cam.right, cam.fwd);
    cam.tan_half = std::tan(0.5 * d->vertical_fov_degrees * M_PI / 180.0);
    cam.aspect = (double)d->width / (double)d->height;
    const double n = 0.1, f = 1000.0;
    double V[4][4] = {{cam.right.x, cam.right.y, cam.right.z, -dot(cam.right, cam.eye)},
                      {cam.up.x, cam.up.y, cam.up.z, -dot(cam.up, cam.eye)},
                      {-cam.fwd.x, -cam.fwd.y, -cam.fwd.z, dot(cam.fwd, cam.eye)},
                      {0, 0, 0, 1}};
    // Projection with the y axis flipped so that image row 0 is the top and
    // pixel row y maps to uv.y = (y + 0.5) / H.
    double P[4][4] = {{1.0 / (cam.aspect * cam.tan_half), 0, 0, 0},
                      {0, -1.0 / cam.tan_half, 0, 0},
                      {0, 0, (f + n) / (n - f), 2.0 * f * n / (n - f)},
                      {0, 0, -1, 0}};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double acc = 0.0;
            for (int k = 0; k < 4; ++k) acc += P[i][k] * V[k][j];
            cam.vp[i][j] = acc;
        }
    return cam;
}

}  // namespace bmfr_scene_internal
