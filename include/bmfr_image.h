/* bmfr_image.h — image output for quality regression (host memory).
 *
 * The reference writes its results as PNG files through OpenImageIO
 * (opencl/bmfr.cpp:527-545); here frames are written and read as Portable
 * Float Maps (PFM: "PF", width height, -1.0 for little-endian, then float
 * RGB rows from the bottom row up), which keep the float values exactly, and
 * compared by PSNR.  Buffers are W*H*3 floats, top row first, as the
 * pipeline's outputs.
 */
#ifndef BMFR_IMAGE_H
#define BMFR_IMAGE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

int bmfr_write_pfm(const char* path, int width, int height, const float* rgb);
/* Reads a colour PFM of at most `capacity` floats; width/height receive its
 * size.  Both byte orders are accepted. */
int bmfr_read_pfm(const char* path, int* width, int* height, float* rgb, size_t capacity);
/* 10 log10(peak^2 / MSE) over n values (+inf for identical inputs). */
double bmfr_psnr(const float* a, const float* b, size_t n, float peak);

#ifdef __cplusplus
}
#endif
#endif /* BMFR_IMAGE_H */
