// vsg_fpchain.h -- exact O(1) replay of the ray caster's FP32 step chain.
//
// The reference marches with rayCurrent += 0.5 * voxelSize in binary32
// (RayCastRender.cu:389-392), so sample k sits at the k-th value of the
// chain r <- RN(r + h), not at r0 + k h.  Skipping provably empty samples
// must land on exactly the value the serial additions would produce.
//
// Within one binade [2^e, 2^(e+1)) every float is an integer multiple of
// u = ulp = 2^(e-23).  Writing r = R u and h = H u (H real), RN(r + h) =
// (R + RN(H)) u as long as the sum stays below 2^(e+1) and H is not a tie
// (odd multiple of 1/2), so the chain advances by the constant D = RN(H)
// ulps: r_k = (R + k D) u, exact in integer arithmetic.  Binade crossings
// and ties fall back to one real FP32 addition.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define VSG_HD __host__ __device__ __forceinline__
#else
#define VSG_HD static inline
#include <math.h>
#include <string.h>
#endif

VSG_HD uint32_t vsg_f2u(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
#endif
}

VSG_HD float vsg_u2f(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
}

// An estimate of x / y for the step count, corrected by exact integer
// comparisons afterwards, so its last bits do not matter.
#ifdef __CUDA_ARCH__
#define VSG_QUOT_EST(x, y) __fdividef((x), (y))
#else
#define VSG_QUOT_EST(x, y) ((x) / (y))
#endif

// 2^k for -126 <= k <= 127
VSG_HD float vsg_pow2(int k) { return vsg_u2f((uint32_t)(k + 127) << 23); }

// Advance r along r <- RN(r + h) to the first chain value >= target.
// Requires h > 0 finite.  *steps receives the number of additions taken;
// at most max_steps are taken (the caller's iteration guard).  Values of r
// that are not positive normal floats, and ties, use plain additions (for
// h = voxel/2 ties never occur in the binades a ray visits).
VSG_HD float vsg_chain_advance(float r, float h, float target, int max_steps, int* steps) {
    int taken = 0;
    // every pass takes at least one step or returns, so max_steps bounds it
    while (r < target && taken < max_steps) {
        const uint32_t bits = vsg_f2u(r);
        const int be = (int)((bits >> 23) & 0xFFu);
        if ((bits >> 31) || be < 24 || be >= 254 - 24) {  // non-positive, tiny or huge: serial step
            r = r + h;
            ++taken;
            continue;
        }
        const int e = be - 127;
        // H = h / u exactly (power-of-two scaling; h / u < 2^24 since h < r
        // unless the chain is at its very start, which the serial path takes)
        if (!(h < r)) {
            r = r + h;
            ++taken;
            continue;
        }
        const float H = h * vsg_pow2(23 - e);
        const float Hf = floorf(H);
        const float frac = H - Hf;
        if (frac == 0.5f) {  // tie: rounding depends on the parity of R
            r = r + h;
            ++taken;
            continue;
        }
        const int D = (int)Hf + (frac > 0.5f ? 1 : 0);
        if (D == 0) {  // r + h rounds back to r: the chain is stuck until max_steps
            taken = max_steps;
            break;
        }
        const int R = (int)(bits & 0x7FFFFFu) | 0x800000;  // r / u
        // steps needed to reach target: smallest k >= 1 with R + k D >= T
        const float T = target * vsg_pow2(23 - e);  // exact scaling
        int kneed;
        if (!(T < 16777216.0f)) {
            kneed = 0x7FFFFFFF;
        } else {
            const float need = T - (float)R;  // an estimate; corrected below
            kneed = (int)ceilf(VSG_QUOT_EST(need, (float)D));
            if (kneed < 1) kneed = 1;
            // correct the float estimate with exact integer comparisons
            while (kneed > 1 && (float)(R + (kneed - 1) * D) >= T) --kneed;
            while ((float)(R + kneed * D) < T) ++kneed;
        }
        const int room = max_steps - taken;
        // R + kneed D <= 2^24 - 2: the kneed steps stay strictly inside the binade
        if (kneed <= room && (long long)R + (long long)kneed * D <= 0xFFFFFE) {
            r = (float)(R + kneed * D) * vsg_pow2(e - 23);
            taken += kneed;
            break;
        }
        // steps that keep R + k D <= 2^24 - 2
        const int kmax = (0xFFFFFE - R) / D;
        int k = kmax < room ? kmax : room;
        if (k > 0) {
            r = (float)(R + k * D) * vsg_pow2(e - 23);
            taken += k;
        }
        if (taken < max_steps && r < target) {
            r = r + h;  // the step that crosses into the next binade
            ++taken;
        }
    }
    if (steps) *steps += taken;
    return r;
}
