// capi.cu — the C ABI of include/bmfr_b200.h: parameter checks, the plan
// (sizes plus the frame pipeline's history buffers) and the launches.
//
// The plan mirrors the reference host program's buffer set and frame loop
// (opencl/bmfr.cpp:315-347, 417-485): six double-buffered histories swapped
// after every frame and eight single buffers, all resident in HBM.
#include "bmfr_b200.h"
#include "kernels.h"
#include "status.h"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace bmfr {

int fail(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(BMFR_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace bmfr

using bmfr::cuda_fail;
using bmfr::fail;

struct bmfr_plan {
    bmfr_params p;
    bmfr::Geometry g;
    int device = 0;
    int frame = 0;
    // Frame-pipeline buffers (bmfr.cpp:315-347).  The plan's input slots
    // are three sets used in turn (set f % 3 for frame f), so that frame
    // f+1 can be uploaded while frame f is denoised, which also reads the
    // normals and positions of frame f-1.
    float* normals[3] = {nullptr, nullptr, nullptr};
    float* positions[3] = {nullptr, nullptr, nullptr};
    float* albedo[3] = {nullptr, nullptr, nullptr};
    float* noisy_in[3] = {nullptr, nullptr, nullptr};   // the frame's 1-spp colour
    void* noisy_acc[2] = {nullptr, nullptr};    // accumulated noisy history
    uint8_t* spp[2] = {nullptr, nullptr};
    // Per-frame buffers that the accumulation writes and only the same
    // frame's later stages read.  Set 1 exists once bmfr_denoise_frames has
    // overlapped frames (frame f then uses set f & 1); otherwise every frame
    // uses set 0.
    struct FrameScratch {
        void* tmp = nullptr;
        float2* prev_pix = nullptr;
        uint8_t* accept = nullptr;
        float* noise_table = nullptr;   // the frame's fitter noise
    } scratch[2];
    int last_set = 0;                   // the set of the last frame
    float* weights = nullptr;
    float* mins_maxs = nullptr;
    float* filtered = nullptr;
    float* tone_mapped = nullptr;
    void* acc_filt[2] = {nullptr, nullptr};     // accumulated filtered history
    void* result[2] = {nullptr, nullptr};       // TAA history
    float* result_f32[2] = {nullptr, nullptr};  // fp32 output when histories are binary16
    int* dev_status = nullptr;                  // device error word (bounded waits)
    const float* last_result = nullptr;         // float32 output of the last frame
    bool profiling = false;
    bool profiled_frame = false;
    bool keep_intermediates = false;            // also write the filtered frame
    cudaEvent_t events[6] = {};                 // stage boundaries of the last frame
    // Ordering of uploads, frames and downloads that run on different
    // streams: input set k uploaded, frame f done (index f % 3), result of
    // parity p read back.  The flags say whether the event was recorded.
    cudaEvent_t ev_uploaded[3] = {}, ev_frame_done[3] = {}, ev_downloaded[2] = {};
    bool uploaded[3] = {}, downloaded[2] = {}, done_recorded[3] = {};
    // bmfr_denoise_frames: the streams that run the accumulations of
    // overlapped frames (lowest priority) and the rest of each frame
    // (highest priority), the end of frame f's accumulation (index f & 1),
    // and the call's entry and exit on the caller's stream.
    cudaStream_t acc_stream = nullptr, frame_stream = nullptr;
    cudaEvent_t ev_accumulated[2] = {}, ev_entry = nullptr, ev_exit = nullptr;
    std::vector<void*> allocations;
};

namespace {

bool check_device(const bmfr_plan* plan) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    return dev == plan->device;
}

int check_plan(const bmfr_plan* plan) {
    if (!plan) return fail(BMFR_E_INVALID, "plan is NULL");
    if (!check_device(plan)) return fail(BMFR_E_STATE, "the current CUDA device is not the plan's device");
    return BMFR_OK;
}

size_t pixel3_bytes(const bmfr_plan* p, bool half) {
    return (size_t)p->g.W * p->g.H * 3 * (half ? 2 : 4);
}

size_t tmp_bytes(const bmfr::Geometry& g, bool half) {
    return (size_t)g.MW * g.MH * bmfr::kBuffers * (half ? 2 : 4);
}

bmfr::AccumArgs accum_args(const bmfr_plan* plan, const float* m, const float* off, int frame) {
    bmfr::AccumArgs a;
    std::memcpy(a.m, m, sizeof a.m);
    a.off_x = off[0];
    a.off_y = off[1];
    a.pos_lim2 = plan->p.position_limit_squared;
    a.nrm_lim2 = plan->p.normal_limit_squared;
    a.blend_alpha = plan->p.blend_alpha;
    a.frame = frame;
    a.use_half = plan->p.use_half_precision_in_tmp_data ? 1 : 0;
    return a;
}

void free_plan(bmfr_plan* plan) {
    for (cudaEvent_t& e : plan->events)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : plan->ev_uploaded)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : plan->ev_frame_done)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : plan->ev_downloaded)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : plan->ev_accumulated)
        if (e) cudaEventDestroy(e);
    if (plan->ev_entry) cudaEventDestroy(plan->ev_entry);
    if (plan->ev_exit) cudaEventDestroy(plan->ev_exit);
    if (plan->acc_stream) cudaStreamDestroy(plan->acc_stream);
    if (plan->frame_stream) cudaStreamDestroy(plan->frame_stream);
    for (void* p : plan->allocations) cudaFree(p);
    delete plan;
}

}  // namespace

extern "C" {

const char* bmfr_last_error(void) { return g_last_error.c_str(); }

const char* bmfr_status_string(int status) {
    switch (status) {
        case BMFR_OK: return "ok";
        case BMFR_E_INVALID: return "invalid argument";
        case BMFR_E_CUDA: return "CUDA error";
        case BMFR_E_UNSUPPORTED: return "unsupported parameter";
        case BMFR_E_NOMEM: return "out of device memory";
        case BMFR_E_BUDGET: return "over the memory budget";
        case BMFR_E_NOT_FOUND: return "not found";
        case BMFR_E_AGAIN: return "not ready";
        case BMFR_E_TIMEOUT: return "timed out";
        case BMFR_E_STATE: return "invalid state";
        case BMFR_E_TOO_LARGE: return "size beyond the fixed maximum";
        default: return "unknown status";
    }
}

int bmfr_params_default(bmfr_params* p) {
    if (!p) return fail(BMFR_E_INVALID, "params is NULL");
    std::memset(p, 0, sizeof *p);
    p->noise_amount = 1e-2;            // bmfr.cpp:58
    p->blend_alpha = 0.2f;             // bmfr.cpp:60
    p->second_blend_alpha = 0.1f;      // bmfr.cpp:61
    p->taa_blend_alpha = 0.2f;         // bmfr.cpp:62
    p->position_limit_squared = 0.01f; // dataset-defined in the reference
    p->normal_limit_squared = 0.1f;
    p->use_half_precision_in_tmp_data = 1;   // bmfr.cpp:88
    p->compressed_r = 1;               // bmfr.cpp:82
    p->cache_tmp_data = 1;             // bmfr.cpp:84
    p->fp32_qr = 0;
    p->half_history = 0;
    p->pipeline = BMFR_PIPELINE_STAGED;
    return BMFR_OK;
}

int bmfr_block_offsets(int out_xy[32]) {
    static const int t[32] = {-14, -14, 4, -6, -8, 14, 8, 0, -10, -8, 2, 12, 12, -12, -10, 0,
                              12, 14, -8, -16, 6, 6, -2, -2, 6, -14, -16, 12, 14, -4, -6, 4};
    if (!out_xy) return fail(BMFR_E_INVALID, "out_xy is NULL");
    std::memcpy(out_xy, t, sizeof t);
    return BMFR_OK;
}

namespace {

// The checks of bmfr_plan_create, for the entry point that takes no plan.
int validate(const bmfr_params* params, int width, int height) {
    if (width < 32 || height < 32 || width > 16384 || height > 16384)
        return fail(BMFR_E_INVALID, "image size must be within [32, 16384]");
    const bmfr::Geometry g = bmfr::make_geometry(width, height);
    // mirror() (bmfr.cl:209-216) must stay within one image size: the margin
    // grid reaches WORKSET + 29 on the right/bottom and -32 on the left/top.
    if (g.MW - 3 > 2 * width - 1 || g.MH - 3 > 2 * height - 1)
        return fail(BMFR_E_UNSUPPORTED, "image too small for the mirrored 16-pixel margin");
    if (!params->cache_tmp_data) return fail(BMFR_E_UNSUPPORTED, "cache_tmp_data = 0 is not served");
    if (params->fp32_qr < 0 || params->fp32_qr > 2) return fail(BMFR_E_INVALID, "fp32_qr must be 0, 1 or 2");
    return BMFR_OK;
}

}  // namespace

int bmfr_plan_create(const bmfr_params* params, int width, int height, bmfr_plan** out) {
    if (!params || !out) return fail(BMFR_E_INVALID, "params/plan pointer is NULL");
    *out = nullptr;
    if (width < 32 || height < 32 || width > 16384 || height > 16384)
        return fail(BMFR_E_INVALID, "image size must be within [32, 16384]");
    const bmfr::Geometry g = bmfr::make_geometry(width, height);
    // mirror() (bmfr.cl:209-216) must stay within one image size: the margin
    // grid reaches WORKSET + 29 on the right/bottom and -32 on the left/top.
    if (g.MW - 3 > 2 * width - 1 || g.MH - 3 > 2 * height - 1)
        return fail(BMFR_E_UNSUPPORTED, "image too small for the mirrored 16-pixel margin");
    if (!params->cache_tmp_data) return fail(BMFR_E_UNSUPPORTED, "cache_tmp_data = 0 is not served");
    if (params->pipeline != BMFR_PIPELINE_STAGED && params->pipeline != BMFR_PIPELINE_FUSED)
        return fail(BMFR_E_INVALID, "unknown pipeline");
    if (params->fp32_qr < 0 || params->fp32_qr > 2) return fail(BMFR_E_INVALID, "fp32_qr must be 0, 1 or 2");
    if (!(params->blend_alpha > 0.f) || !(params->second_blend_alpha > 0.f))
        return fail(BMFR_E_INVALID, "blend factors must be positive");
    int device = -1;
    if (cudaError_t e = cudaGetDevice(&device); e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(e, "no CUDA device");
    }
    bmfr_plan* plan = new bmfr_plan;
    plan->p = *params;
    plan->g = g;
    plan->device = device;
    const bool half_tmp = params->use_half_precision_in_tmp_data != 0;
    const bool half_hist = params->half_history != 0;
    const size_t px = (size_t)width * height;
    auto alloc = [&](size_t bytes, auto** ptr) -> bool {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        cudaMemset(p, 0, bytes);
        plan->allocations.push_back(p);
        *ptr = static_cast<std::remove_pointer_t<decltype(ptr)>>(p);
        return true;
    };
    bool ok = true;
    for (int i = 0; i < 3 && ok; ++i)
        ok = alloc(px * 12, &plan->normals[i]) && alloc(px * 12, &plan->positions[i]) &&
             alloc(px * 12, &plan->albedo[i]) && alloc(px * 12, &plan->noisy_in[i]);
    for (int i = 0; i < 2 && ok; ++i) {
        ok = ok && alloc(pixel3_bytes(plan, half_hist), &plan->noisy_acc[i]) && alloc(px, &plan->spp[i]) &&
             alloc(pixel3_bytes(plan, half_hist), &plan->acc_filt[i]) &&
             alloc(pixel3_bytes(plan, half_hist), &plan->result[i]);
        if (ok && half_hist) ok = alloc(px * 12, &plan->result_f32[i]);
    }
    bmfr_plan::FrameScratch& fs = plan->scratch[0];
    ok = ok && alloc(tmp_bytes(g, half_tmp), &fs.tmp) &&
         alloc((size_t)g.blocks * bmfr::kFeatures * 3 * 4, &plan->weights) &&
         alloc((size_t)g.blocks * bmfr::kScaled * 2 * 4, &plan->mins_maxs) &&
         alloc(px * 12, &plan->filtered) && alloc(px * 8, &fs.prev_pix) && alloc(px, &fs.accept) &&
         alloc(px * 12, &plan->tone_mapped);
    if (ok) ok = alloc(sizeof(int), &plan->dev_status) && alloc(bmfr::kNoiseTableBytes, &fs.noise_table);
    for (int i = 0; i < 3 && ok; ++i)
        ok = cudaEventCreateWithFlags(&plan->ev_uploaded[i], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&plan->ev_frame_done[i], cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < 2 && ok; ++i)
        ok = cudaEventCreateWithFlags(&plan->ev_downloaded[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        free_plan(plan);
        return fail(BMFR_E_NOMEM, "device allocation for the plan failed");
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        free_plan(plan);
        return cuda_fail(e, "plan initialisation");
    }
    *out = plan;
    return BMFR_OK;
}

int bmfr_plan_destroy(bmfr_plan* plan) {
    if (!plan) return BMFR_OK;
    free_plan(plan);
    return BMFR_OK;
}

int bmfr_plan_sizes(const bmfr_plan* plan, bmfr_sizes* s) {
    if (!plan || !s) return fail(BMFR_E_INVALID, "NULL argument");
    const bmfr::Geometry& g = plan->g;
    s->image_width = g.W;
    s->image_height = g.H;
    s->workset_width = g.MW - 32;
    s->workset_height = g.MH - 32;
    s->margin_width = g.MW;
    s->margin_height = g.MH;
    s->blocks_x = g.MWb;
    s->blocks_y = g.MHb;
    s->blocks = g.blocks;
    s->tmp_data_bytes = tmp_bytes(g, plan->p.use_half_precision_in_tmp_data != 0);
    s->weights_bytes = (size_t)g.blocks * bmfr::kFeatures * 3 * sizeof(float);
    s->mins_maxs_bytes = (size_t)g.blocks * bmfr::kScaled * 2 * sizeof(float);
    s->pixel3_bytes = (size_t)g.W * g.H * 3 * sizeof(float);
    return BMFR_OK;
}

int bmfr_plan_params(const bmfr_plan* plan, bmfr_params* p) {
    if (!plan || !p) return fail(BMFR_E_INVALID, "NULL argument");
    *p = plan->p;
    return BMFR_OK;
}

int bmfr_accumulate_noisy_data(const bmfr_plan* plan, float* out_prev_frame_pixel, uint8_t* accept_bools,
                               const float* current_normals, const float* previous_normals,
                               const float* current_positions, const float* previous_positions,
                               float* current_noisy, const float* previous_noisy, const uint8_t* previous_spp,
                               uint8_t* current_spp, void* tmp_data, const float* prev_frame_camera_matrix,
                               const float* pixel_offset, int frame_number, void* stream) {
    if (int st = check_plan(plan)) return st;
    if (!out_prev_frame_pixel || !accept_bools || !current_normals || !current_positions || !current_noisy ||
        !current_spp || !tmp_data || !prev_frame_camera_matrix || !pixel_offset)
        return fail(BMFR_E_INVALID, "accumulate_noisy_data: NULL buffer");
    if (frame_number < 0) return fail(BMFR_E_INVALID, "accumulate_noisy_data: negative frame number");
    if (frame_number > 0 && (!previous_normals || !previous_positions || !previous_noisy || !previous_spp))
        return fail(BMFR_E_INVALID, "accumulate_noisy_data: NULL history buffer");
    const bmfr::AccumArgs a = accum_args(plan, prev_frame_camera_matrix, pixel_offset, frame_number);
    cudaError_t e = bmfr::launch_accumulate_noisy(
        plan->g, a, reinterpret_cast<float2*>(out_prev_frame_pixel), accept_bools, current_normals,
        previous_normals, current_positions, previous_positions, current_noisy, current_noisy, previous_noisy,
        false, previous_spp, current_spp, tmp_data, (cudaStream_t)stream);
    return e == cudaSuccess ? BMFR_OK : cuda_fail(e, "accumulate_noisy_data launch");
}

int bmfr_fitter(const bmfr_plan* plan, float* weights, float* mins_maxs, const void* tmp_data, int frame_number,
                void* stream) {
    if (int st = check_plan(plan)) return st;
    if (!weights || !mins_maxs || !tmp_data) return fail(BMFR_E_INVALID, "fitter: NULL buffer");
    if (reinterpret_cast<uintptr_t>(tmp_data) % 16 != 0)
        return fail(BMFR_E_INVALID, "fitter: tmp_data must be 16-byte aligned");
    if (frame_number < 0) return fail(BMFR_E_INVALID, "fitter: negative frame number");
    cudaError_t e = bmfr::launch_fitter(plan->g, frame_number, bmfr::make_noise_const(plan->p.noise_amount),
                                        tmp_data, plan->p.use_half_precision_in_tmp_data != 0,
                                        plan->p.fp32_qr, weights, mins_maxs, nullptr, plan->dev_status,
                                        (cudaStream_t)stream);
    return e == cudaSuccess ? BMFR_OK : cuda_fail(e, "fitter launch");
}

int bmfr_fitter_fp64(const bmfr_plan* plan, double* weights, float* mins_maxs, const void* tmp_data,
                     int frame_number, void* stream) {
    if (int st = check_plan(plan)) return st;
    if (!weights || !mins_maxs || !tmp_data) return fail(BMFR_E_INVALID, "fitter_fp64: NULL buffer");
    if (frame_number < 0) return fail(BMFR_E_INVALID, "fitter_fp64: negative frame number");
    cudaError_t e = bmfr::launch_fitter_fp64(plan->g, frame_number, plan->p.noise_amount, tmp_data,
                                             plan->p.use_half_precision_in_tmp_data != 0, weights, mins_maxs,
                                             (cudaStream_t)stream);
    return e == cudaSuccess ? BMFR_OK : cuda_fail(e, "fitter_fp64 launch");
}

int bmfr_fitter_noalloc(const bmfr_params* params, int width, int height, float* weights, float* mins_maxs,
                        const void* tmp_data, int frame_number, void* stream) {
    if (!params) return fail(BMFR_E_INVALID, "fitter_noalloc: params is NULL");
    if (int st = validate(params, width, height)) return st;
    if (!weights || !mins_maxs || !tmp_data) return fail(BMFR_E_INVALID, "fitter_noalloc: NULL buffer");
    if (reinterpret_cast<uintptr_t>(tmp_data) % 16 != 0)
        return fail(BMFR_E_INVALID, "fitter_noalloc: tmp_data must be 16-byte aligned");
    if (frame_number < 0) return fail(BMFR_E_INVALID, "fitter_noalloc: negative frame number");
    const bmfr::Geometry g = bmfr::make_geometry(width, height);
    cudaError_t e = bmfr::launch_fitter_static(g, frame_number, bmfr::make_noise_const(params->noise_amount),
                                               tmp_data, params->use_half_precision_in_tmp_data != 0,
                                               params->fp32_qr, weights, mins_maxs, (cudaStream_t)stream);
    return e == cudaSuccess ? BMFR_OK : cuda_fail(e, "fitter_noalloc launch");
}

int bmfr_fitter_noalloc_check(void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    int* status = nullptr;
    cudaError_t e = bmfr::static_fitter_status(&status, s);
    if (e != cudaSuccess) return cuda_fail(e, "fitter_noalloc_check");
    int v = 0;
    e = cudaMemcpyAsync(&v, status, sizeof v, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "fitter_noalloc_check");
    if (v != 0) {
        e = cudaMemsetAsync(status, 0, sizeof(int), s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(e, "fitter_noalloc_check");
        return fail(BMFR_E_TIMEOUT, "a bmfr_fitter_noalloc kernel's bounded wait ran out (device status " +
                                        std::to_string(v) + ")");
    }
    return BMFR_OK;
}

int bmfr_fitter_noalloc_probe_bounded_wait(unsigned int limit_us, void* stream) {
    if (limit_us < 1 || limit_us > 1000000) return fail(BMFR_E_INVALID, "limit_us must be within [1, 1000000]");
    cudaStream_t s = (cudaStream_t)stream;
    int* status = nullptr;
    cudaError_t e = bmfr::static_fitter_status(&status, s);
    if (e == cudaSuccess) e = bmfr::launch_bounded_wait_probe(status, 1000ull * limit_us, s);
    return e == cudaSuccess ? BMFR_OK : cuda_fail(e, "fitter_noalloc_probe_bounded_wait");
}

int bmfr_weighted_sum(const bmfr_plan* plan, const float* weights, const float* mins_maxs, float* output,
                      const float* current_normals, const float* current_positions, const float* current_noisy,
                      int frame_number, void* stream) {
    (void)current_noisy;   // debug-only in the reference (bmfr.cl:709, 752-754)
    if (int st = check_plan(plan)) return st;
    if (!weights || !mins_maxs || !output || !current_normals || !current_positions)
        return fail(BMFR_E_INVALID, "weighted_sum: NULL buffer");
    if (frame_number < 0) return fail(BMFR_E_INVALID, "weighted_sum: negative frame number");
    cudaError_t e = bmfr::launch_weighted_sum(plan->g, frame_number, weights, mins_maxs, output, current_normals,
                                              current_positions, (cudaStream_t)stream);
    return e == cudaSuccess ? BMFR_OK : cuda_fail(e, "weighted_sum launch");
}

int bmfr_accumulate_filtered_data(const bmfr_plan* plan, const float* filtered_frame,
                                  const float* in_prev_frame_pixel, const uint8_t* accept_bools,
                                  const float* albedo, float* tone_mapped_frame, const uint8_t* current_spp,
                                  const float* accumulated_prev_frame, float* accumulated_frame, int frame_number,
                                  void* stream) {
    if (int st = check_plan(plan)) return st;
    if (!filtered_frame || !albedo || !tone_mapped_frame || !accumulated_frame)
        return fail(BMFR_E_INVALID, "accumulate_filtered_data: NULL buffer");
    if (frame_number < 0) return fail(BMFR_E_INVALID, "accumulate_filtered_data: negative frame number");
    if (frame_number > 0 && (!in_prev_frame_pixel || !accept_bools || !current_spp || !accumulated_prev_frame))
        return fail(BMFR_E_INVALID, "accumulate_filtered_data: NULL history buffer");
    cudaError_t e = bmfr::launch_accumulate_filtered(
        plan->g, frame_number, plan->p.second_blend_alpha, filtered_frame,
        reinterpret_cast<const float2*>(in_prev_frame_pixel), accept_bools, albedo, tone_mapped_frame,
        current_spp, accumulated_prev_frame, accumulated_frame, (cudaStream_t)stream);
    return e == cudaSuccess ? BMFR_OK : cuda_fail(e, "accumulate_filtered_data launch");
}

int bmfr_taa(const bmfr_plan* plan, const float* in_prev_frame_pixel, const float* new_frame, float* result_frame,
             const float* prev_frame, int frame_number, void* stream) {
    if (int st = check_plan(plan)) return st;
    if (!in_prev_frame_pixel || !new_frame || !result_frame) return fail(BMFR_E_INVALID, "taa: NULL buffer");
    if (frame_number < 0) return fail(BMFR_E_INVALID, "taa: negative frame number");
    if (frame_number > 0 && !prev_frame) return fail(BMFR_E_INVALID, "taa: NULL history buffer");
    cudaError_t e = bmfr::launch_taa(plan->g, frame_number, plan->p.taa_blend_alpha,
                                     reinterpret_cast<const float2*>(in_prev_frame_pixel), new_frame, result_frame,
                                     prev_frame, nullptr, false, (cudaStream_t)stream);
    return e == cudaSuccess ? BMFR_OK : cuda_fail(e, "taa launch");
}

// ---- plan-managed pipeline ------------------------------------------------

int bmfr_plan_frame_inputs(bmfr_plan* plan, bmfr_frame_inputs* in) {
    if (!plan || !in) return fail(BMFR_E_INVALID, "NULL argument");
    const int k = plan->frame % 3;
    in->albedo = plan->albedo[k];
    in->normals = plan->normals[k];
    in->positions = plan->positions[k];
    in->noisy = plan->noisy_in[k];
    return BMFR_OK;
}

int bmfr_plan_upload_frame(bmfr_plan* plan, const float* albedo, const float* normals, const float* positions,
                           const float* noisy, void* stream) {
    if (int st = check_plan(plan)) return st;
    if (!albedo || !normals || !positions || !noisy) return fail(BMFR_E_INVALID, "upload: NULL host buffer");
    bmfr_frame_inputs in;
    bmfr_plan_frame_inputs(plan, &in);
    const int f = plan->frame, k = f % 3;
    const size_t bytes = (size_t)plan->g.W * plan->g.H * 12;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    // Set k was last read by frame f-2 (its previous normals and positions);
    // the first two frames (after a reset too) wait for every frame recorded.
    if (f >= 2) {
        e = cudaStreamWaitEvent(s, plan->ev_frame_done[(f - 2) % 3], 0);
    } else {
        for (int i = 0; i < 3 && e == cudaSuccess; ++i)
            if (plan->done_recorded[i]) e = cudaStreamWaitEvent(s, plan->ev_frame_done[i], 0);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(in.albedo, albedo, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(in.normals, normals, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(in.positions, positions, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(in.noisy, noisy, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(plan->ev_uploaded[k], s);
    if (e != cudaSuccess) return cuda_fail(e, "upload");
    plan->uploaded[k] = true;
    return BMFR_OK;
}

namespace {

// One frame of the pipeline (bmfr.cpp:429-476) on the given inputs; the
// histories are the plan's.  prev_n/prev_p may be null at frame 0.  The
// frame's noise table and accumulation run on `sa` (the plan's accumulation
// stream while bmfr_denoise_frames overlaps frames, else `s`) into per-frame
// buffer set `set`; everything after them runs on `s`.
int run_frame(bmfr_plan* plan, const float* albedo, const float* cur_n, const float* prev_n, const float* cur_p,
              const float* prev_p, const float* noisy, float* extra_result, const float* m, const float* off,
              cudaStream_t s, cudaStream_t sa = nullptr, int set = 0) {
    const int f = plan->frame;
    const int cur = f & 1, prv = cur ^ 1;
    const bmfr::Geometry& g = plan->g;
    const bool half_tmp = plan->p.use_half_precision_in_tmp_data != 0;
    const bool half_hist = plan->p.half_history != 0;
    // The fused pipeline accumulates inside its block kernel: never split.
    const bool split = sa != nullptr && sa != s && plan->p.pipeline == BMFR_PIPELINE_STAGED;
    if (!split) sa = s;
    const bmfr_plan::FrameScratch& fs = plan->scratch[set];
    if (f > 0 && (!prev_n || !prev_p)) return fail(BMFR_E_INVALID, "denoise_frame: previous G-buffer missing");
    const bmfr::AccumArgs a = accum_args(plan, m, off, f);
    const bool prof = plan->profiling && !split;
    auto mark = [&](int i) {
        if (prof) cudaEventRecord(plan->events[i], s);
    };
    cudaError_t e = cudaSuccess;
    // Uploads and downloads may run on other streams: wait for this frame's
    // input set (read first by the accumulation; the later stages are
    // ordered after it) and for the read-back of the result buffers this
    // frame overwrites (those of frame f-2).
    if (plan->uploaded[f % 3] && albedo == plan->albedo[f % 3]) {
        e = cudaStreamWaitEvent(sa, plan->ev_uploaded[f % 3], 0);
        plan->uploaded[f % 3] = false;
    }
    if (e == cudaSuccess && plan->downloaded[cur]) {
        e = cudaStreamWaitEvent(s, plan->ev_downloaded[cur], 0);
        plan->downloaded[cur] = false;
    }
    mark(0);
    if (e == cudaSuccess) e = bmfr::launch_noise_table(f, fs.noise_table, sa);
    if (plan->p.pipeline == BMFR_PIPELINE_FUSED) {
        mark(1);
        bmfr::FusedBuffers fb;
        fb.cur_n = cur_n;
        fb.prev_n = prev_n;
        fb.cur_p = cur_p;
        fb.prev_p = prev_p;
        fb.noisy_in = noisy;
        fb.albedo = albedo;
        fb.noisy_acc_cur = plan->noisy_acc[cur];
        fb.noisy_acc_prev = plan->noisy_acc[prv];
        fb.prev_spp = plan->spp[prv];
        fb.cur_spp = plan->spp[cur];
        fb.prev_pix = fs.prev_pix;
        fb.accept = fs.accept;
        fb.tone_mapped = plan->tone_mapped;
        fb.acc_prev = plan->acc_filt[prv];
        fb.acc_cur = plan->acc_filt[cur];
        fb.weights = plan->weights;
        fb.mins_maxs = plan->mins_maxs;
        fb.noise = fs.noise_table;
        if (e == cudaSuccess)
            e = bmfr::launch_fused_block(g, a, bmfr::make_noise_const(plan->p.noise_amount),
                                         plan->p.second_blend_alpha, plan->p.fp32_qr, half_hist, fb, false, s);
        mark(2);
    } else {
        if (e == cudaSuccess)
            e = bmfr::launch_accumulate_noisy(g, a, fs.prev_pix, fs.accept, cur_n, prev_n, cur_p, prev_p, noisy,
                                              plan->noisy_acc[cur], plan->noisy_acc[prv], half_hist, plan->spp[prv],
                                              plan->spp[cur], fs.tmp, sa);
        mark(1);
        // The rest of the frame waits for its accumulation only.
        if (e == cudaSuccess && split) e = cudaEventRecord(plan->ev_accumulated[cur], sa);
        if (e == cudaSuccess && split) e = cudaStreamWaitEvent(s, plan->ev_accumulated[cur], 0);
        if (e == cudaSuccess)
            e = bmfr::launch_fitter(g, f, bmfr::make_noise_const(plan->p.noise_amount), fs.tmp, half_tmp,
                                    plan->p.fp32_qr, plan->weights, plan->mins_maxs, fs.noise_table,
                                    plan->dev_status, s);
        mark(2);
    }
    // weighted_sum and accumulate_filtered_data in one pass per pixel; the
    // filtered colour is written only when kept for inspection
    // (bmfr_plan_keep_intermediates).
    if (e == cudaSuccess)
        e = bmfr::launch_weighted_sum_accumulate(g, f, plan->p.second_blend_alpha, plan->weights, plan->mins_maxs,
                                                 cur_n, cur_p, plan->keep_intermediates ? plan->filtered : nullptr,
                                                 fs.prev_pix, fs.accept, albedo, plan->tone_mapped,
                                                 plan->spp[cur], plan->acc_filt[prv], plan->acc_filt[cur], half_hist,
                                                 s);
    mark(3);
    mark(4);
    float* f32_out = extra_result ? extra_result : (half_hist ? plan->result_f32[cur] : nullptr);
    if (e == cudaSuccess)
        e = bmfr::launch_taa(g, f, plan->p.taa_blend_alpha, fs.prev_pix, plan->tone_mapped, plan->result[cur],
                             plan->result[prv], f32_out, half_hist, s);
    mark(5);
    if (e == cudaSuccess) e = cudaEventRecord(plan->ev_frame_done[f % 3], s);
    if (e != cudaSuccess) return cuda_fail(e, "denoise_frame launch");
    plan->done_recorded[f % 3] = true;
    plan->profiled_frame = prof;
    plan->last_set = set;
    plan->last_result = half_hist ? f32_out : (const float*)plan->result[cur];
    plan->frame = f + 1;   // swaps every double buffer (bmfr.cpp:482-484)
    return BMFR_OK;
}

// The second set of per-frame buffers, the two streams and their events,
// made by the first call that overlaps frames.  Set 1 is published only when
// all of it exists.  The accumulation of frame f+1 has the length of frame
// f's later stages as slack, so its stream has the lowest priority and the
// other the highest: the block scheduler then gives free SM slots to the
// fitter, weighted sum and TAA first, and the accumulation takes the slots
// they leave (mostly in the fitter's last wave).
int ensure_overlap_resources(bmfr_plan* plan, cudaStream_t s) {
    if (plan->scratch[1].tmp) return BMFR_OK;
    const size_t px = (size_t)plan->g.W * plan->g.H;
    bmfr_plan::FrameScratch fs;
    const size_t bytes[4] = {tmp_bytes(plan->g, plan->p.use_half_precision_in_tmp_data != 0), px * 8, px,
                             bmfr::kNoiseTableBytes};
    void* ptr[4] = {};
    for (int i = 0; i < 4; ++i) {
        if (cudaMalloc(&ptr[i], bytes[i]) != cudaSuccess) {
            cudaGetLastError();
            return fail(BMFR_E_NOMEM, "device allocation for overlapped frames failed");
        }
        plan->allocations.push_back(ptr[i]);
        cudaError_t e = cudaMemsetAsync(ptr[i], 0, bytes[i], s);
        if (e != cudaSuccess) return cuda_fail(e, "overlapped frames: buffer initialisation");
    }
    int least = 0, greatest = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess && !plan->acc_stream)
        e = cudaStreamCreateWithPriority(&plan->acc_stream, cudaStreamNonBlocking, least);
    if (e == cudaSuccess && !plan->frame_stream)
        e = cudaStreamCreateWithPriority(&plan->frame_stream, cudaStreamNonBlocking, greatest);
    for (int i = 0; i < 2 && e == cudaSuccess; ++i)
        if (!plan->ev_accumulated[i]) e = cudaEventCreateWithFlags(&plan->ev_accumulated[i], cudaEventDisableTiming);
    if (e == cudaSuccess && !plan->ev_entry) e = cudaEventCreateWithFlags(&plan->ev_entry, cudaEventDisableTiming);
    if (e == cudaSuccess && !plan->ev_exit) e = cudaEventCreateWithFlags(&plan->ev_exit, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(e, "overlapped frames: stream and events");
    fs.tmp = ptr[0];
    fs.prev_pix = static_cast<float2*>(ptr[1]);
    fs.accept = static_cast<uint8_t*>(ptr[2]);
    fs.noise_table = static_cast<float*>(ptr[3]);
    plan->scratch[1] = fs;
    return BMFR_OK;
}

}  // namespace

int bmfr_denoise_frame(bmfr_plan* plan, const float* prev_frame_camera_matrix, const float* pixel_offset,
                       void* stream) {
    if (int st = check_plan(plan)) return st;
    if (!prev_frame_camera_matrix || !pixel_offset) return fail(BMFR_E_INVALID, "denoise_frame: NULL matrix/offset");
    const int k = plan->frame % 3, kp = (plan->frame + 2) % 3;
    return run_frame(plan, plan->albedo[k], plan->normals[k], plan->normals[kp], plan->positions[k],
                     plan->positions[kp], plan->noisy_in[k], nullptr, prev_frame_camera_matrix, pixel_offset,
                     (cudaStream_t)stream);
}

int bmfr_denoise_frame_io(bmfr_plan* plan, const bmfr_frame_io* io, const float* prev_frame_camera_matrix,
                          const float* pixel_offset, void* stream) {
    if (int st = check_plan(plan)) return st;
    if (!io || !prev_frame_camera_matrix || !pixel_offset)
        return fail(BMFR_E_INVALID, "denoise_frame_io: NULL argument");
    if (!io->albedo || !io->normals || !io->positions || !io->noisy)
        return fail(BMFR_E_INVALID, "denoise_frame_io: NULL input buffer");
    return run_frame(plan, io->albedo, io->normals, io->previous_normals, io->positions, io->previous_positions,
                     io->noisy, io->result, prev_frame_camera_matrix, pixel_offset, (cudaStream_t)stream);
}

int bmfr_denoise_frames(bmfr_plan* plan, int count, const bmfr_frame_io* io, const float* prev_frame_camera_matrices,
                        const float* pixel_offsets, void* stream) {
    if (int st = check_plan(plan)) return st;
    if (count < 0) return fail(BMFR_E_INVALID, "denoise_frames: negative count");
    if (count == 0) return BMFR_OK;
    if (!io || !prev_frame_camera_matrices || !pixel_offsets)
        return fail(BMFR_E_INVALID, "denoise_frames: NULL argument");
    // Every frame is checked before the first is queued, so a bad entry
    // leaves the plan where it was.
    for (int i = 0; i < count; ++i) {
        const bmfr_frame_io& x = io[i];
        if (!x.albedo || !x.normals || !x.positions || !x.noisy)
            return fail(BMFR_E_INVALID, "denoise_frames: NULL input buffer in io[" + std::to_string(i) + "]");
        if (plan->frame + i > 0 && (!x.previous_normals || !x.previous_positions))
            return fail(BMFR_E_INVALID, "denoise_frames: previous G-buffer missing in io[" + std::to_string(i) + "]");
    }
    cudaStream_t caller = (cudaStream_t)stream, s = caller;
    const bool overlap = count > 1 && plan->p.pipeline == BMFR_PIPELINE_STAGED && !plan->profiling;
    cudaStream_t sa = nullptr;
    if (overlap) {
        if (int st = ensure_overlap_resources(plan, caller)) return st;
        sa = plan->acc_stream;
        s = plan->frame_stream;
        // Both streams start after the work already on the caller's stream.
        cudaError_t e = cudaEventRecord(plan->ev_entry, caller);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(sa, plan->ev_entry, 0);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, plan->ev_entry, 0);
        if (e != cudaSuccess) return cuda_fail(e, "denoise_frames: entry");
    }
    // On an error part way through, whatever was queued on the two streams
    // is still ordered before the caller's later work (best effort: the
    // error being returned is the one that counts).
    auto join_on_error = [&]() {
        if (!overlap) return;
        if (cudaEventRecord(plan->ev_exit, s) == cudaSuccess) cudaStreamWaitEvent(caller, plan->ev_exit, 0);
        if (cudaEventRecord(plan->ev_entry, sa) == cudaSuccess) cudaStreamWaitEvent(caller, plan->ev_entry, 0);
    };
    for (int i = 0; i < count; ++i) {
        const bmfr_frame_io& x = io[i];
        const int f = plan->frame;
        // Frame f's accumulation rewrites the per-frame buffers and the spp
        // history that frame f-2 read on `stream`; frame f-1 uses the other
        // set, and its accumulation precedes this one on the same stream.
        if (overlap && i >= 2) {
            cudaError_t e = cudaStreamWaitEvent(sa, plan->ev_frame_done[(f - 2) % 3], 0);
            if (e != cudaSuccess) {
                join_on_error();
                return cuda_fail(e, "denoise_frames: frame order");
            }
        }
        if (int st = run_frame(plan, x.albedo, x.normals, x.previous_normals, x.positions, x.previous_positions,
                               x.noisy, x.result, prev_frame_camera_matrices + 16 * (size_t)i,
                               pixel_offsets + 2 * (size_t)i, s, sa, overlap ? (f & 1) : 0)) {
            join_on_error();
            return st;
        }
    }
    if (overlap) {
        // Every accumulation has been waited for on the frame stream; its
        // last TAA ends the call on the caller's stream.
        cudaError_t e = cudaEventRecord(plan->ev_exit, s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(caller, plan->ev_exit, 0);
        if (e != cudaSuccess) return cuda_fail(e, "denoise_frames: exit");
    }
    return BMFR_OK;
}

int bmfr_plan_result(const bmfr_plan* plan, const float** result) {
    if (!plan || !result) return fail(BMFR_E_INVALID, "NULL argument");
    if (plan->frame == 0) return fail(BMFR_E_STATE, "no frame has been denoised");
    *result = plan->last_result;
    return BMFR_OK;
}

int bmfr_plan_download_result(bmfr_plan* plan, float* host_rgb, void* stream) {
    if (int st = check_plan(plan)) return st;
    if (!host_rgb) return fail(BMFR_E_INVALID, "download: NULL host buffer");
    const float* r = nullptr;
    if (int st = bmfr_plan_result(plan, &r)) return st;
    const int f = plan->frame - 1;   // the last denoised frame
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaStreamWaitEvent(s, plan->ev_frame_done[f % 3], 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(host_rgb, r, (size_t)plan->g.W * plan->g.H * 12, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaEventRecord(plan->ev_downloaded[f & 1], s);
    if (e != cudaSuccess) return cuda_fail(e, "download");
    plan->downloaded[f & 1] = true;
    return BMFR_OK;
}

int bmfr_plan_frame_number(const bmfr_plan* plan) { return plan ? plan->frame : BMFR_E_INVALID; }

int bmfr_plan_reset(bmfr_plan* plan) {
    if (!plan) return fail(BMFR_E_INVALID, "plan is NULL");
    plan->frame = 0;
    plan->last_result = nullptr;
    return BMFR_OK;
}

int bmfr_plan_check_device(const bmfr_plan* plan, void* stream) {
    if (int st = check_plan(plan)) return st;
    int v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, plan->dev_status, sizeof v, cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "check_device");
    if (v != 0) {
        cudaMemsetAsync(plan->dev_status, 0, sizeof(int), (cudaStream_t)stream);
        cudaStreamSynchronize((cudaStream_t)stream);
        return fail(BMFR_E_TIMEOUT, "a kernel's bounded wait ran out (device status " + std::to_string(v) + ")");
    }
    return BMFR_OK;
}

int bmfr_plan_probe_bounded_wait(bmfr_plan* plan, unsigned int limit_us, void* stream) {
    if (int st = check_plan(plan)) return st;
    if (limit_us < 1 || limit_us > 1000000) return fail(BMFR_E_INVALID, "limit_us must be within [1, 1000000]");
    const cudaError_t e = bmfr::launch_bounded_wait_probe(plan->dev_status, 1000ull * limit_us,
                                                          (cudaStream_t)stream);
    return e == cudaSuccess ? BMFR_OK : cuda_fail(e, "probe_bounded_wait");
}

int bmfr_plan_keep_intermediates(bmfr_plan* plan, int enable) {
    if (int st = check_plan(plan)) return st;
    plan->keep_intermediates = enable != 0;
    return BMFR_OK;
}

int bmfr_plan_enable_profiling(bmfr_plan* plan, int enable) {
    if (int st = check_plan(plan)) return st;
    if (enable && !plan->events[0]) {
        for (cudaEvent_t& e : plan->events) {
            cudaError_t r = cudaEventCreate(&e);
            if (r != cudaSuccess) return cuda_fail(r, "cudaEventCreate");
        }
    }
    plan->profiling = enable != 0;
    return BMFR_OK;
}

int bmfr_plan_stage_times(const bmfr_plan* plan, float ms[BMFR_STAGE_COUNT]) {
    if (int st = check_plan(plan)) return st;
    if (!ms) return fail(BMFR_E_INVALID, "ms is NULL");
    if (!plan->profiled_frame) return fail(BMFR_E_STATE, "no profiled frame");
    cudaError_t e = cudaEventSynchronize(plan->events[5]);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventSynchronize");
    for (int i = 0; i < BMFR_STAGE_COUNT; ++i) {
        e = cudaEventElapsedTime(&ms[i], plan->events[i], plan->events[i + 1]);
        if (e != cudaSuccess) return cuda_fail(e, "cudaEventElapsedTime");
    }
    return BMFR_OK;
}

int bmfr_plan_buffers_get(const bmfr_plan* plan, bmfr_plan_buffers* b) {
    if (!plan || !b) return fail(BMFR_E_INVALID, "NULL argument");
    std::memset(b, 0, sizeof *b);
    const int last = (plan->frame + 1) & 1;   // slot written by the last frame
    const bool staged = plan->p.pipeline == BMFR_PIPELINE_STAGED;
    const bmfr_plan::FrameScratch& fs = plan->scratch[plan->last_set];
    b->tmp_data = staged ? fs.tmp : nullptr;   // the fused pipeline keeps tmp_data on chip
    b->weights = plan->weights;
    b->mins_maxs = plan->mins_maxs;
    b->filtered = plan->keep_intermediates ? plan->filtered : nullptr;
    b->prev_frame_pixel = reinterpret_cast<const float*>(fs.prev_pix);
    b->tone_mapped = plan->tone_mapped;
    b->accept = fs.accept;
    b->spp = plan->spp[last];
    b->accumulated_noisy = plan->noisy_acc[last];
    b->accumulated_filtered = plan->acc_filt[last];
    b->result = plan->last_result;
    return BMFR_OK;
}

}  // extern "C"
