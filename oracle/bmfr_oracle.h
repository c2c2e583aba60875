/* bmfr_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's five OpenCL kernels (opencl/bmfr.cl),
 * used as the parity checker of the CUDA pipeline and as the timed CPU
 * baseline.  Nothing in the product links or calls this library.
 *
 * PINNED to the reference itself: the reference's own kernels (opencl/bmfr.cl)
 * are compiled for the CPU by oracle/ref_cl (g++ through an OpenCL C
 * compatibility header, a fiber per work-item) and every output of this
 * restatement equals theirs bit for bit, intermediates included
 * (tests/test_reference_pin.py; fixtures in tests/golden/).
 *
 * All buffers are HOST memory with the reference's layouts.
 */
#ifndef BMFR_ORACLE_H
#define BMFR_ORACLE_H
#include <stdint.h>
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_cfg {
    int width, height;
    double noise_amount;           /* NOISE_AMOUNT, a double literal (bmfr.cpp:58) */
    float blend_alpha, second_blend_alpha, taa_blend_alpha;
    float position_limit_squared, normal_limit_squared;
    int use_half;                  /* tmp_data binary16 (1) or float32 (0)   */
    int threads;                   /* OpenMP threads; <= 0: all              */
} orc_cfg;

/* Fitter arithmetic modes. */
#define ORC_FITTER_REFERENCE 0  /* fp32, every tmp store rounded to the tmp type */
#define ORC_FITTER_FP32 1       /* fp32 QR, no intermediate rounding            */
#define ORC_FITTER_FP64 2       /* fp64 QR, no intermediate rounding            */

void orc_sizes(const orc_cfg* cfg, int* margin_w, int* margin_h, int* blocks);

/* bmfr.cl:290-485.  current_noisy is in/out (the blended colour replaces the
 * input for in-image pixels); mirrored margin pixels see the raw input. */
void orc_accumulate_noisy_data(const orc_cfg* cfg, float* out_prev_frame_pixel,
    uint8_t* accept_bools, const float* current_normals,
    const float* previous_normals, const float* current_positions,
    const float* previous_positions, float* current_noisy,
    const float* previous_noisy, const uint8_t* previous_spp,
    uint8_t* current_spp, void* tmp_data, const float* camera_matrix,
    const float* pixel_offset, int frame_number);

/* bmfr.cl:490-700.  tmp_data is modified in place as in the reference. */
void orc_fitter(const orc_cfg* cfg, float* weights, float* mins_maxs,
    void* tmp_data, int frame_number, int mode);

/* Double-precision outputs of the fp64 fitter mode (weights as doubles). */
void orc_fitter_fp64(const orc_cfg* cfg, double* weights, float* mins_maxs,
    const void* tmp_data, int frame_number);

/* The least-squares system every block solves: for each block, its 13
 * columns of 1024 values after the min/max scaling and the noise of the
 * first column step, in double precision (out: blocks x 13 x 1024). */
void orc_fitter_matrix(const orc_cfg* cfg, const void* tmp_data, int frame_number,
    double* out);

void orc_weighted_sum(const orc_cfg* cfg, const float* weights,
    const float* mins_maxs, float* output, const float* current_normals,
    const float* current_positions, int frame_number);

void orc_accumulate_filtered_data(const orc_cfg* cfg, const float* filtered_frame,
    const float* in_prev_frame_pixel, const uint8_t* accept_bools,
    const float* albedo, float* tone_mapped_frame, const uint8_t* current_spp,
    const float* accumulated_prev_frame, float* accumulated_frame,
    int frame_number);

void orc_taa(const orc_cfg* cfg, const float* in_prev_frame_pixel,
    const float* new_frame, float* result_frame, const float* prev_frame,
    int frame_number);

/* Small helpers exposed for known-answer tests. */
float orc_random(uint32_t a);                 /* bmfr.cl:162-171 */
int orc_mirror(int index, int size);          /* bmfr.cl:209-216 */
float orc_round_half(float v);                /* vstore_half, round to nearest even */
float orc_add_random(float value, int id, int sub_vector, int feature_buffer,
                     int frame_number, double noise_amount);  /* bmfr.cl:173-182 */

#ifdef __cplusplus
}
#endif
#endif
