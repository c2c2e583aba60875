// image.cu — PFM output and PSNR (include/bmfr_image.h), host code only.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "bmfr_b200.h"
#include "bmfr_image.h"
#include "status.h"

using bmfr::fail;

namespace {

bool host_little_endian() {
    const uint16_t v = 1;
    unsigned char c;
    std::memcpy(&c, &v, 1);
    return c == 1;
}

float byteswap(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u = (u >> 24) | ((u >> 8) & 0xff00u) | ((u << 8) & 0xff0000u) | (u << 24);
    std::memcpy(&f, &u, 4);
    return f;
}

}  // namespace

extern "C" {

int bmfr_write_pfm(const char* path, int width, int height, const float* rgb) {
    if (!path || !rgb || width <= 0 || height <= 0) return fail(BMFR_E_INVALID, "write_pfm: bad argument");
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(BMFR_E_INVALID, std::string("write_pfm: cannot open ") + path);
    const bool le = host_little_endian();
    std::fprintf(f, "PF\n%d %d\n%s\n", width, height, le ? "-1.0" : "1.0");
    bool ok = true;
    for (int y = height - 1; y >= 0 && ok; --y)   // PFM rows run bottom to top
        ok = std::fwrite(rgb + (size_t)y * width * 3, sizeof(float), (size_t)width * 3, f) == (size_t)width * 3;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? BMFR_OK : fail(BMFR_E_INVALID, std::string("write_pfm: writing ") + path + " failed");
}

int bmfr_read_pfm(const char* path, int* width, int* height, float* rgb, size_t capacity) {
    if (!path || !width || !height) return fail(BMFR_E_INVALID, "read_pfm: bad argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(BMFR_E_NOT_FOUND, std::string("read_pfm: cannot open ") + path);
    char tag[3] = {0, 0, 0};
    int w = 0, h = 0;
    double scale = 0.0;
    const bool header = std::fscanf(f, "%2s %d %d %lf", tag, &w, &h, &scale) == 4 && std::strcmp(tag, "PF") == 0 &&
                        w > 0 && h > 0 && scale != 0.0 && std::fgetc(f) != EOF;
    if (!header) {
        std::fclose(f);
        return fail(BMFR_E_INVALID, "read_pfm: not a colour PFM");
    }
    *width = w;
    *height = h;
    const size_t n = (size_t)w * h * 3;
    if (!rgb) {
        std::fclose(f);
        return BMFR_OK;   // size query
    }
    if (capacity < n) {
        std::fclose(f);
        return fail(BMFR_E_TOO_LARGE, "read_pfm: buffer too small");
    }
    bool ok = true;
    for (int y = h - 1; y >= 0 && ok; --y)
        ok = std::fread(rgb + (size_t)y * w * 3, sizeof(float), (size_t)w * 3, f) == (size_t)w * 3;
    std::fclose(f);
    if (!ok) return fail(BMFR_E_INVALID, "read_pfm: file too short");
    if ((scale < 0.0) != host_little_endian())
        for (size_t i = 0; i < n; ++i) rgb[i] = byteswap(rgb[i]);
    return BMFR_OK;
}

double bmfr_psnr(const float* a, const float* b, size_t n, float peak) {
    if (!a || !b || n == 0) return std::numeric_limits<double>::quiet_NaN();
    double se = 0.0;
    for (size_t i = 0; i < n; ++i) {
        const double d = (double)a[i] - (double)b[i];
        se += d * d;
    }
    if (se == 0.0) return std::numeric_limits<double>::infinity();
    const double mse = se / (double)n;
    return 10.0 * std::log10((double)peak * (double)peak / mse);
}

}  // extern "C"
