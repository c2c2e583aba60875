/* Checks, on the host, the quotient sequence the fitter kernels use for
 * a / b (fit_block.cuh: qr_column and scale_by):
 *     y = RN(1/b);  q0 = RN(a*y);  r = fma(-q0, b, a);  q = -fma(-r, y, -q0)
 * against IEEE division, over random operands whose magnitudes stay inside
 * the ranges the kernels admit to this path (|a| in [2^-64, 2^60] or 0,
 * b in [2^-60, 2^60]), including divisors with all-ones significands and
 * signed zeros.  Prints the number of mismatches (must be 0). */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static uint64_t s = 0x9e3779b97f4a7c15ull;
static uint64_t next(void) { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; }
static float from_bits(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static uint32_t bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

static float markstein(float a, float b) {
    const float y = 1.0f / b;
    const float q0 = a * y;
    const float r = fmaf(-q0, b, a);
    return -fmaf(-r, y, -q0);
}

int main(int argc, char** argv) {
    long n = argc > 1 ? atol(argv[1]) : 1000000;
    long bad = 0;
    for (long i = 0; i < n; ++i) {
        uint32_t ea = 63 + next() % 124, eb = 67 + next() % 121;   /* 2^-64..2^60, 2^-60..2^60 */
        uint32_t ua = (ea << 23) | (next() & 0x7fffff) | ((uint32_t)(next() & 1) << 31);
        uint32_t ub = (eb << 23) | (next() & 0x7fffff);
        if (i % 7 == 0) ub = (eb << 23) | 0x7fffff;
        if (i % 11 == 0) ub = (eb << 23) | (0x7fffff - (next() & 15));
        if (i % 13 == 0) ua = (ua & 0x80000000u);   /* signed zero numerator */
        const float a = from_bits(ua), b = from_bits(ub);
        const float q = markstein(a, b), ref = a / b;
        if (bits(q) != bits(ref)) {
            if (bad < 5) printf("mismatch a=%a b=%a got=%a want=%a\n", a, b, q, ref);
            ++bad;
        }
    }
    printf("%ld\n", bad);
    return bad != 0;
}
