// ref_runner.cpp — TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own OpenCL kernels (opencl/bmfr.cl, prepared by
// prepare.py and compiled by g++ against cl_compat.h) on the CPU, launched the
// way the reference host program launches them (opencl/bmfr.cpp:245-249,
// 417-476), with the compile-time options it passes (bmfr.cpp:193-232).  The
// library built from this file (oracle/_ref/libbmfr_ref.so) pins the oracle
// restatement (oracle/bmfr_oracle.cpp): both take the same orc_cfg and host
// buffers, and the tests require their outputs to be identical.
//
// Execution model (a minimal CPU OpenCL runtime for these five kernels).  A
// kernel without barriers runs its work-items as plain calls, rows of the
// NDRange spread over OpenMP threads.  The fitter (barriers, __local memory)
// runs each work-group's 256 work-items as fibers of one thread, work-groups
// spread over OpenMP threads: every barrier switches to the next fiber, so
// all work-items of the group reach the barrier before any passes it.  Kernel-scope __local
// variables are `static thread_local`, i.e. one per group in flight.
//
// accumulate_noisy_data reads current_noisy at mirrored margin pixels while
// in-image work-items overwrite it in place (bmfr.cl:322, :481): the
// kernel's result depends on the order of its work-items.  The runner runs
// the margin work-items first, a legal order in which every mirrored read
// sees the colour as it was before the kernel — the semantics the oracle
// defines for that race.
#include "cl_compat.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../bmfr_oracle.h"

namespace clc {

// ---- run-time values of the reference's -D options ---------------------------
struct RunParams {
    int image_width, image_height;
    int workset_width, workset_height;
    int margins_width, margins_height;
    double noise_amount;
    float blend_alpha, second_blend_alpha, taa_blend_alpha;
    float position_limit_squared, normal_limit_squared;
};
static RunParams rt;

}  // namespace clc

// bmfr.cpp:206-232.  The fixed options are literals as there; the options the
// host computes from the image size or reads from its configuration are
// variables set per call.
#define BUFFER_COUNT 13
#define FEATURES_NOT_SCALED 4
#define FEATURES_SCALED 6
#define IMAGE_WIDTH (clc::rt.image_width)
#define IMAGE_HEIGHT (clc::rt.image_height)
#define WORKSET_WIDTH (clc::rt.workset_width)
#define WORKSET_HEIGHT (clc::rt.workset_height)
// bmfr.cpp:65-77 (NOT_SCALED_FEATURE_BUFFERS SCALED_FEATURE_BUFFERS)
#define FEATURE_BUFFERS 1.f, normal.x, normal.y, normal.z, world_position.x, world_position.y, \
    world_position.z, world_position.x*world_position.x, world_position.y*world_position.y, \
    world_position.z*world_position.z
#define LOCAL_WIDTH 8
#define LOCAL_HEIGHT 8
#define WORKSET_WITH_MARGINS_WIDTH (clc::rt.margins_width)
#define WORKSET_WITH_MARGINS_HEIGHT (clc::rt.margins_height)
#define BLOCK_EDGE_LENGTH 32
#define BLOCK_PIXELS 1024
#define R_EDGE 11
#define NOISE_AMOUNT (clc::rt.noise_amount)
#define BLEND_ALPHA (clc::rt.blend_alpha)
#define SECOND_BLEND_ALPHA (clc::rt.second_blend_alpha)
#define TAA_BLEND_ALPHA (clc::rt.taa_blend_alpha)
#define POSITION_LIMIT_SQUARED (clc::rt.position_limit_squared)
#define NORMAL_LIMIT_SQUARED (clc::rt.normal_limit_squared)
#define COMPRESSED_R 1
#define CACHE_TMP_DATA 1
#define ADD_REQD_WG_SIZE 1
#define LOCAL_SIZE 256

// The kernel source, once with binary16 tmp_data (the reference's setting,
// bmfr.cpp:88) and once with float32.
namespace clc { namespace k16 {
#define USE_HALF_PRECISION_IN_TMP_DATA 1
#include "bmfr_cl.inc"
#undef USE_HALF_PRECISION_IN_TMP_DATA
}}
#undef BLOCK_EDGE_HALF
#undef HORIZONTAL_BLOCKS
#undef BLOCK_INDEX_X
#undef BLOCK_INDEX_Y
#undef IN_BLOCK_INDEX
#undef FEATURE_START
#undef IN_ACCESS
#undef R_SIZE
#undef R_ROW_START
#undef R_ACCESS
#undef load_float3
#undef LOAD
#undef STORE
#undef BLOCK_OFFSETS_COUNT
namespace clc { namespace k32 {
#define USE_HALF_PRECISION_IN_TMP_DATA 0
#include "bmfr_cl.inc"
#undef USE_HALF_PRECISION_IN_TMP_DATA
}}

namespace clc {

thread_local const WorkItem* tl_item = nullptr;

// ---- fibers: one work-group at a time per thread --------------------------------
// A fiber switch saves the callee-saved general registers of the x86-64
// System V ABI (rbx, rbp, r12-r15) on the running stack, stores the stack
// pointer and loads the other one.  MXCSR and the x87 control word are not
// switched: nothing here changes them, so every fiber runs with the thread's
// settings.  (glibc's swapcontext also saves the signal mask, a system call
// per switch.)
extern "C" void clc_fiber_switch(void** save_sp, void* load_sp);
__asm__(
    ".text\n"
    ".p2align 4\n"
    ".globl clc_fiber_switch\n"
    ".hidden clc_fiber_switch\n"
    ".type clc_fiber_switch,@function\n"
    "clc_fiber_switch:\n"
    "  pushq %rbp\n"
    "  pushq %rbx\n"
    "  pushq %r12\n"
    "  pushq %r13\n"
    "  pushq %r14\n"
    "  pushq %r15\n"
    "  movq %rsp, (%rdi)\n"
    "  movq %rsi, %rsp\n"
    "  popq %r15\n"
    "  popq %r14\n"
    "  popq %r13\n"
    "  popq %r12\n"
    "  popq %rbx\n"
    "  popq %rbp\n"
    "  ret\n"
    ".size clc_fiber_switch, .-clc_fiber_switch\n");

namespace {

constexpr int kGroupSize = 256;            // LOCAL_SIZE
constexpr size_t kStackBytes = 16 * 1024;

struct Fiber {
    void* sp;
    WorkItem item;
    bool done;
};

struct FiberPool {
    std::vector<Fiber> fibers;
    std::vector<uint64_t> stacks;          // 8-byte words, 16-byte aligned slices
    void* scheduler_sp = nullptr;
    Fiber* current = nullptr;
    void (*body)(void*) = nullptr;
    void* arg = nullptr;
    bool active = false;
};
thread_local FiberPool tl_pool;

[[noreturn]] void fiber_entry() {
    FiberPool& p = tl_pool;
    p.body(p.arg);
    p.current->done = true;
    clc_fiber_switch(&p.current->sp, p.scheduler_sp);   // never resumed
    std::abort();
}

// The first switch into a fiber pops the frame built here: six zero
// registers, then `ret` enters fiber_entry with the stack aligned as after a
// call.
void* initial_frame(uint64_t* top) {
    uint64_t* sp = top;
    *--sp = 0;                                               // fiber_entry's return address (unused)
    *--sp = reinterpret_cast<uint64_t>(&fiber_entry);
    for (int i = 0; i < 6; ++i) *--sp = 0;                   // rbp rbx r12 r13 r14 r15
    return sp;
}

// Runs one work-group of the 1-D NDRange: `body(arg)` once per work-item, as
// fibers that switch at every barrier.
bool run_group(size_t group, void (*body)(void*), void* arg) {
    FiberPool& p = tl_pool;
    constexpr size_t words = kStackBytes / 8;
    if (p.fibers.empty()) {
        p.fibers.resize(kGroupSize);
        p.stacks.resize(words * kGroupSize + 2);
    }
    uint64_t* base = p.stacks.data();
    base += (reinterpret_cast<uintptr_t>(base) & 15) ? 1 : 0;   // 16-byte aligned tops
    p.body = body;
    p.arg = arg;
    p.active = true;
    for (int i = 0; i < kGroupSize; ++i) {
        Fiber& f = p.fibers[i];
        f.done = false;
        f.item = WorkItem{{group * kGroupSize + i, 0, 0}, {(size_t)i, 0, 0}, {group, 0, 0}};
        // Tops staggered by 7 cache lines per fiber: equal offsets in 16 KB
        // slices would map every fiber's live frame to the same cache sets.
        f.sp = initial_frame(base + words * (i + 1) - (size_t)((i * 56) % 512));
    }
    bool ok = true;
    for (;;) {
        int done = 0, waiting = 0;
        for (int i = 0; i < kGroupSize; ++i) {
            Fiber& f = p.fibers[i];
            if (f.done) { ++done; continue; }
            p.current = &f;
            tl_item = &f.item;
            clc_fiber_switch(&p.scheduler_sp, f.sp);
            if (f.done) ++done; else ++waiting;
        }
        if (waiting == 0) break;
        if (done != 0) {          // some work-items ended while others wait at a barrier
            ok = false;
            break;
        }
    }
    p.active = false;
    tl_item = nullptr;
    return ok;
}

}  // namespace

void barrier_yield() {
    FiberPool& p = tl_pool;
    if (!p.active) {
        std::fprintf(stderr, "ref_runner: barrier outside a fiber work-group\n");
        std::abort();
    }
    Fiber* f = p.current;
    clc_fiber_switch(&f->sp, p.scheduler_sp);
}

// ---- NDRange helpers ---------------------------------------------------------------
static int threads_of(const orc_cfg* cfg) {
#ifdef _OPENMP
    return cfg->threads > 0 ? cfg->threads : omp_get_max_threads();
#else
    (void)cfg;
    return 1;
#endif
}

static void set_params(const orc_cfg* cfg) {
    rt.image_width = cfg->width;
    rt.image_height = cfg->height;
    rt.workset_width = 32 * ((cfg->width + 31) / 32);     // bmfr.cpp:107-110
    rt.workset_height = 32 * ((cfg->height + 31) / 32);
    rt.margins_width = rt.workset_width + 32;             // bmfr.cpp:111-112
    rt.margins_height = rt.workset_height + 32;
    rt.noise_amount = cfg->noise_amount;
    rt.blend_alpha = cfg->blend_alpha;
    rt.second_blend_alpha = cfg->second_blend_alpha;
    rt.taa_blend_alpha = cfg->taa_blend_alpha;
    rt.position_limit_squared = cfg->position_limit_squared;
    rt.normal_limit_squared = cfg->normal_limit_squared;
}

// A 2-D NDRange without barriers: `f(x, y)` for the work-items with keep(x, y).
template <class F, class Keep>
static void run_2d(const orc_cfg* cfg, int gx, int gy, F f, Keep keep) {
    const int nt = threads_of(cfg);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int y = 0; y < gy; ++y) {
        WorkItem wi{};
        for (int x = 0; x < gx; ++x) {
            if (!keep(x, y)) continue;
            wi.global_id[0] = (size_t)x;
            wi.global_id[1] = (size_t)y;
            wi.local_id[0] = (size_t)(x % LOCAL_WIDTH);
            wi.local_id[1] = (size_t)(y % LOCAL_HEIGHT);
            wi.group_id[0] = (size_t)(x / LOCAL_WIDTH);
            wi.group_id[1] = (size_t)(y / LOCAL_HEIGHT);
            tl_item = &wi;
            f();
        }
        tl_item = nullptr;
    }
}

}  // namespace clc

using namespace clc;

namespace {

struct FitterArgs {
    bool half;
    float* weights;
    float* mins_maxs;
    void* tmp;
    int frame;
};

thread_local std::vector<float> tl_sum_vec, tl_u_vec;
thread_local std::vector<float3> tl_r_mat;

void fitter_item(void* a) {
    const FitterArgs& f = *static_cast<const FitterArgs*>(a);
    if (f.half)
        k16::fitter(tl_sum_vec.data(), tl_u_vec.data(), tl_r_mat.data(), f.weights, f.mins_maxs,
                    static_cast<half*>(f.tmp), f.frame);
    else
        k32::fitter(tl_sum_vec.data(), tl_u_vec.data(), tl_r_mat.data(), f.weights, f.mins_maxs,
                    static_cast<float*>(f.tmp), f.frame);
}

}  // namespace

extern "C" {

// bmfr.cl:290-485, NDRange (WORKSET_WITH_MARGINS_WIDTH, _HEIGHT) / (8, 8)
// (bmfr.cpp:245, 247, 446).
int ref_accumulate_noisy_data(const orc_cfg* cfg, float* out_prev_frame_pixel, uint8_t* accept_bools,
                              const float* current_normals, const float* previous_normals,
                              const float* current_positions, const float* previous_positions,
                              float* current_noisy, const float* previous_noisy, const uint8_t* previous_spp,
                              uint8_t* current_spp, void* tmp_data, const float* camera_matrix,
                              const float* pixel_offset, int frame_number) {
    set_params(cfg);
    float16 m;
    std::memcpy(m.s, camera_matrix, sizeof(m.s));
    const float2 off(pixel_offset[0], pixel_offset[1]);
    float2* ppix = reinterpret_cast<float2*>(out_prev_frame_pixel);
    const int W = cfg->width, H = cfg->height;
    const int ox = -16 + k16::BLOCK_OFFSETS[frame_number % 16].x;
    const int oy = -16 + k16::BLOCK_OFFSETS[frame_number % 16].y;
    auto outside = [=](int x, int y) {
        const int px = x + ox, py = y + oy;
        return px < 0 || px >= W || py < 0 || py >= H;
    };
    auto run = [&]() {
        if (cfg->use_half)
            k16::accumulate_noisy_data(ppix, accept_bools, current_normals, previous_normals, current_positions,
                                       previous_positions, current_noisy, previous_noisy, previous_spp,
                                       current_spp, static_cast<half*>(tmp_data), m, off, frame_number);
        else
            k32::accumulate_noisy_data(ppix, accept_bools, current_normals, previous_normals, current_positions,
                                       previous_positions, current_noisy, previous_noisy, previous_spp,
                                       current_spp, static_cast<float*>(tmp_data), m, off, frame_number);
    };
    // Margin work-items (mirrored reads) first, then the in-image ones.
    run_2d(cfg, rt.margins_width, rt.margins_height, run, outside);
    run_2d(cfg, rt.margins_width, rt.margins_height, run, [&](int x, int y) { return !outside(x, y); });
    return 0;
}

// bmfr.cl:490-700, NDRange FITTER_GLOBAL / 256 (bmfr.cpp:116-118, 248-249, 452),
// __local arguments sized as bmfr.cpp:353-363.  Returns 0, or -1 if a
// work-group's work-items did not meet at the same barriers.
int ref_fitter(const orc_cfg* cfg, float* weights, float* mins_maxs, void* tmp_data, int frame_number) {
    set_params(cfg);
    const int groups = (rt.margins_width / 32) * (rt.margins_height / 32);
    const FitterArgs args{cfg->use_half != 0, weights, mins_maxs, tmp_data, frame_number};
    int bad = 0;
    const int nt = threads_of(cfg);
#pragma omp parallel num_threads(nt) reduction(+ : bad)
    {
        tl_sum_vec.assign(LOCAL_SIZE, 0.0f);
        tl_u_vec.assign(BLOCK_PIXELS, 0.0f);
        tl_r_mat.assign((R_EDGE * (R_EDGE + 1)) / 2, float3(0.0f));   // COMPRESSED_R
#pragma omp for schedule(dynamic, 1)
        for (int g = 0; g < groups; ++g) {
            FitterArgs a = args;
            if (!run_group((size_t)g, fitter_item, &a)) ++bad;
        }
    }
    return bad ? -1 : 0;
}

// bmfr.cl:703-758, NDRange (WORKSET_WIDTH, WORKSET_HEIGHT) / (8, 8) (bmfr.cpp:246, 456).
int ref_weighted_sum(const orc_cfg* cfg, const float* weights, const float* mins_maxs, float* output,
                     const float* current_normals, const float* current_positions, int frame_number) {
    set_params(cfg);
    auto run = [&]() {
        k16::weighted_sum(weights, mins_maxs, output, current_normals, current_positions, nullptr, frame_number);
    };
    run_2d(cfg, rt.workset_width, rt.workset_height, run, [](int, int) { return true; });
    return 0;
}

// bmfr.cl:761-857 (bmfr.cpp:463).
int ref_accumulate_filtered_data(const orc_cfg* cfg, const float* filtered_frame, const float* in_prev_frame_pixel,
                                 const uint8_t* accept_bools, const float* albedo, float* tone_mapped_frame,
                                 const uint8_t* current_spp, const float* accumulated_prev_frame,
                                 float* accumulated_frame, int frame_number) {
    set_params(cfg);
    const float2* ppix = reinterpret_cast<const float2*>(in_prev_frame_pixel);
    auto run = [&]() {
        k16::accumulate_filtered_data(filtered_frame, ppix, accept_bools, albedo, tone_mapped_frame, current_spp,
                                      accumulated_prev_frame, accumulated_frame, frame_number);
    };
    run_2d(cfg, rt.workset_width, rt.workset_height, run, [](int, int) { return true; });
    return 0;
}

// bmfr.cl:860-974 (bmfr.cpp:470).
int ref_taa(const orc_cfg* cfg, const float* in_prev_frame_pixel, const float* new_frame, float* result_frame,
            const float* prev_frame, int frame_number) {
    set_params(cfg);
    const float2* ppix = reinterpret_cast<const float2*>(in_prev_frame_pixel);
    auto run = [&]() { k16::taa(ppix, new_frame, result_frame, prev_frame, frame_number); };
    run_2d(cfg, rt.workset_width, rt.workset_height, run, [](int, int) { return true; });
    return 0;
}

}  // extern "C"
