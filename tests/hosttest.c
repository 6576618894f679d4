/* Host build of the library's header-only helpers for CPU unit tests (tests
 * load this through ctypes; the device library compiles the same headers),
 * plus host restatements of device arithmetic that the tests check. */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "vsg_fpchain.h"

float vsg_test_chain_advance(float r, float h, float target, int max_steps, int* steps) {
    *steps = 0;
    return vsg_chain_advance(r, h, target, max_steps, steps);
}

/* reference: serial additions */
float vsg_test_chain_serial(float r, float h, float target, int max_steps, int* steps) {
    int n = 0;
    while (r < target && n < max_steps) {
        r = r + h;
        ++n;
    }
    *steps = n;
    return r;
}

#include "vsg_mc_table.h"

/* the marching-cubes table the kernel uses, 256 x 16 bytes */
void vsg_test_mc_table(unsigned char* out) { vsg_mc_build_table((unsigned char(*)[16])out); }

/* every case generated by the table's geometric rule, 256 x 16 bytes */
void vsg_test_mc_generated(unsigned char* out) { vsg_mc_generate_table((unsigned char(*)[16])out); }

/* The running average's one-correction quotient (avg_div in the device
 * header), restated with the C library's correctly rounded fmaf: for the
 * divisor d and every `stride`-th dividend x in [1, 2), count the x where
 * RN(q + r y), q = RN(x y), r = x - q d, y = RN(1/d), differs from RN(x / d). */
long vsg_test_avg_div_mismatches(int d, int stride) {
    const float df = (float)d, y = 1.0f / df;
    long bad = 0;
    uint32_t m;
    for (m = 0; m < (1u << 23); m += (uint32_t)stride) {
        const uint32_t u = 0x3F800000u | m;
        float x, q, r, z, w;
        memcpy(&x, &u, 4);
        q = x * y;
        r = fmaf(-q, df, x);
        z = fmaf(r, y, q);
        w = x / df;
        bad += memcmp(&z, &w, 4) != 0;
    }
    return bad;
}

/* The smallest float D >= 0 with RN(sqrt(D)) >= w (the integration's
 * squared-distance threshold, sqrt_threshold in the device header),
 * restated with the C library's correctly rounded sqrtf: stepped from
 * RN(w * w), else found by bisection over the float order. */
static float bits_f(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}
static uint32_t f_bits(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}
float vsg_test_sqrt_threshold(float w) {
    float c;
    int i, ok = 0;
    if (!(w > 0.0f) || w == INFINITY) return w;
    c = w * w;
    if (w >= 0x1p-60f && w <= 0x1p60f) {
        for (i = 0; i < 8 && sqrtf(c) < w; ++i) c = bits_f(f_bits(c) + 1u);
        for (i = 0; i < 8 && c > 0.0f && sqrtf(bits_f(f_bits(c) - 1u)) >= w; ++i) c = bits_f(f_bits(c) - 1u);
        ok = sqrtf(c) >= w && (c == 0.0f || sqrtf(bits_f(f_bits(c) - 1u)) < w);
    }
    if (!ok) {
        uint32_t lo = 0u, hi = 0x7F800000u;
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2u;
            if (sqrtf(bits_f(mid)) >= w)
                hi = mid;
            else
                lo = mid + 1u;
        }
        c = bits_f(lo);
    }
    return c;
}
