/* bmfr_scene.h — seeded procedural G-buffer source for the BMFR pipeline.
 *
 * The reference reads 60 frames of EXR feature buffers (world position,
 * shading normal, albedo, 1-spp colour) with OpenImageIO
 * (opencl/bmfr.cpp:145-172, 252-307) and its per-frame view-projection
 * matrices and pixel offsets from the dataset header camera_matrices.h
 * (opencl/bmfr.cpp:44-53, 440-444).  Neither the dataset nor the header is
 * available, so this library renders an equivalent input stream: a ground
 * plane y=0 plus spheres under one directional light, seen by an orbiting
 * camera.  Buffers come out in the reference's interleaved float3 layout.
 *
 * All buffers here are HOST memory; rendering runs on the host cores.
 */
#ifndef BMFR_SCENE_H
#define BMFR_SCENE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bmfr_scene_desc {
    uint64_t seed;
    int width, height;
    int sphere_count;              /* spheres: radius U[0.3,1.5], centre U[-5,5]^2 on y=0 */
    float orbit_degrees_per_frame; /* 0.5 */
    float orbit_start_degrees;
    float orbit_radius;            /* 10 */
    float camera_height;           /* 3 */
    float vertical_fov_degrees;    /* 60 */
    float noise_mu, noise_sigma;   /* lognormal radiance noise, -0.5 / 1.0 */
    float firefly_fraction;        /* 0.001 */
    float firefly_scale;           /* 100 */
    float plane_half_extent;       /* 64: keeps |p|^2 inside binary16 range */
    float position_limit_squared;  /* reprojection limits recorded for the  */
    float normal_limit_squared;    /*   pipeline (bmfr.cpp:226-227)          */
} bmfr_scene_desc;

/* Fills the defaults above for the given seed, size and sphere count. */
int bmfr_scene_default(bmfr_scene_desc* desc, uint64_t seed, int width, int height,
                       int sphere_count);

/* View-projection of frame f in the layout of camera_matrices[f][4][4]
 * (row-vector convention: clip.x = sum_i M[4i+0] * p_i, bmfr.cl:343-347). */
int bmfr_scene_camera(const bmfr_scene_desc* desc, int frame, float matrix[16]);
/* pixel_offsets[f]: (0.5, 0.5) for every frame (no jitter). */
int bmfr_scene_pixel_offset(const bmfr_scene_desc* desc, int frame, float offset[2]);

/* Renders frame f.  noisy is the 1-spp radiance with the albedo divided out
 * ((max(0, n.l) + 0.1) * X, X lognormal, fireflies), which the pipeline
 * multiplies back by albedo after filtering (bmfr.cl:851-854).  clean, if not
 * NULL, receives the noise-free image albedo * (max(0, n.l) + 0.1) after the
 * pipeline's tone map, for PSNR.  Missed pixels are all zero.  threads <= 0
 * uses every host core. */
int bmfr_scene_render(const bmfr_scene_desc* desc, int frame, float* albedo,
                      float* normals, float* positions, float* noisy, float* clean,
                      int threads);

/* The same frame rendered on the current CUDA device into DEVICE buffers:
 * same scene, camera and noise model as bmfr_scene_render in float
 * arithmetic, so values agree to float rounding away from object
 * silhouettes, where a grazing ray may hit a different object.
 * Asynchronous on `stream` (a cudaStream_t).  At most 64 spheres. */
int bmfr_scene_render_device(const bmfr_scene_desc* desc, int frame, float* albedo,
                             float* normals, float* positions, float* noisy, float* clean,
                             void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BMFR_SCENE_H */
