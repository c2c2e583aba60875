// host_loop.cpp — the reference host's frame loop (opencl/bmfr.cpp:417-485)
// as a C++ program written against the C ABI alone, the way the reference's
// host code would call this library: a plan in place of the OpenCL buffers
// and kernels (bmfr.cpp:315-384), host buffers in through
// bmfr_plan_upload_frame, the denoised frame back through
// bmfr_plan_download_result, everything on the legacy default stream (the
// reference's single in-order queue, bmfr.cpp:191).  The inputs are the
// procedural scene of libbmfr_scene, the stand-in for the reference's
// dataset.  Every frame's output is appended to OUT as raw float32 (H x W x
// 3), so a test can compare it with the library's other entry points.
//
// usage: host_loop WIDTH HEIGHT FRAMES SEED OUT
// exit status: 0 done, 2 a library call failed (message on stderr), 64 usage.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "bmfr_b200.h"
#include "bmfr_scene.h"

namespace {

void check(int status, const char* what) {
    if (status == BMFR_OK) return;
    std::fprintf(stderr, "%s: %s (%s)\n", what, bmfr_status_string(status), bmfr_last_error());
    std::exit(2);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s WIDTH HEIGHT FRAMES SEED OUT\n", argv[0]);
        return 64;
    }
    const int width = std::atoi(argv[1]), height = std::atoi(argv[2]), frames = std::atoi(argv[3]);
    const unsigned long long seed = std::strtoull(argv[4], nullptr, 10);

    bmfr_scene_desc scene;
    if (bmfr_scene_default(&scene, seed, width, height, 12) != 0) {
        std::fprintf(stderr, "bmfr_scene_default failed\n");
        return 2;
    }
    // The reference's -D options (bmfr.cpp:205-232) with the dataset's
    // reprojection limits (bmfr.cpp:226-227).
    bmfr_params params;
    check(bmfr_params_default(&params), "bmfr_params_default");
    params.position_limit_squared = scene.position_limit_squared;
    params.normal_limit_squared = scene.normal_limit_squared;
    bmfr_plan* plan = nullptr;
    check(bmfr_plan_create(&params, width, height, &plan), "bmfr_plan_create");

    const size_t n = (size_t)width * height * 3;
    std::vector<float> albedo(n), normals(n), positions(n), noisy(n), result(n);
    std::FILE* out = std::fopen(argv[5], "wb");
    if (!out) {
        std::fprintf(stderr, "cannot open %s\n", argv[5]);
        return 2;
    }
    for (int f = 0; f < frames; ++f) {
        if (bmfr_scene_render(&scene, f, albedo.data(), normals.data(), positions.data(), noisy.data(), nullptr,
                              0) != 0) {
            std::fprintf(stderr, "bmfr_scene_render failed at frame %d\n", f);
            return 2;
        }
        // The matrix of frame f is camera_matrices[max(f-1, 0)], the offset
        // pixel_offsets[f] (bmfr.cpp:440-444).
        float matrix[16], offset[2];
        if (bmfr_scene_camera(&scene, f > 0 ? f - 1 : 0, matrix) != 0 ||
            bmfr_scene_pixel_offset(&scene, f, offset) != 0) {
            std::fprintf(stderr, "scene camera failed at frame %d\n", f);
            return 2;
        }
        check(bmfr_plan_upload_frame(plan, albedo.data(), normals.data(), positions.data(), noisy.data(), nullptr),
              "bmfr_plan_upload_frame");
        check(bmfr_denoise_frame(plan, matrix, offset, nullptr), "bmfr_denoise_frame");
        // A device-to-pageable-host copy returns once the copy is done.
        check(bmfr_plan_download_result(plan, result.data(), nullptr), "bmfr_plan_download_result");
        if (std::fwrite(result.data(), sizeof(float), n, out) != n) {
            std::fprintf(stderr, "write failed at frame %d\n", f);
            return 2;
        }
    }
    std::fclose(out);
    check(bmfr_plan_check_device(plan, nullptr), "bmfr_plan_check_device");
    check(bmfr_plan_destroy(plan), "bmfr_plan_destroy");
    std::printf("%d frames of %dx%d\n", frames, width, height);
    return 0;
}
