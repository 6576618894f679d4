// vsg_raycast_core.cuh -- device code of the ray caster, shared by the
// per-scene kernel (vsg_raycast.cu) and the batched kernel (vsg_batch.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/vsg.h"
#include "vsg_device.cuh"
#include "vsg_fpchain.h"

namespace vsg {

constexpr int kMaxMarch = 1 << 22;  // iteration guard of one ray

struct RenderArgs {
    SceneDev s;
    uint8_t* touched;  // non-null in instrumented runs: mark every block a tap reads
    int W, H;
    float camx, camy, camz;
    Pose pose;
    const float* pose_dev;
    float fx, fy, cx, cy, minD, maxD;
    float* depth;
    float4* pos;
    float4* col;
    float4* nrm;
    float2* rec;  // non-null when recording: per pixel the march bracket of its last zero crossing
};

// Pool indices of the blocks holding a sample's 8 trilinear taps.  The taps
// of one sample span at most two blocks per axis (tap voxels x0 <= x1 <=
// x0 + 2); tp[i] is the block of tap i.  Consecutive samples mostly reuse
// the same blocks, so the entry is kept across samples.
struct TapCache {
    int bx, by, bz, span;
    int t0, t1, t2, t3, t4, t5, t6, t7;
    __device__ __forceinline__ int get(int i) const {
        return i == 0 ? t0 : i == 1 ? t1 : i == 2 ? t2 : i == 3 ? t3 : i == 4 ? t4 : i == 5 ? t5 : i == 6 ? t6 : t7;
    }
    __device__ __forceinline__ void set(int i, int v) {
        if (i == 0) t0 = v; else if (i == 1) t1 = v; else if (i == 2) t2 = v; else if (i == 3) t3 = v;
        else if (i == 4) t4 = v; else if (i == 5) t5 = v; else if (i == 6) t6 = v; else t7 = v;
    }
};

// worldToVirtualVoxelPos, RayCastRender.cu:17-25 (floorf variant)
static __device__ __forceinline__ int tap_voxel(float q) {
    const float sg = (q > 0) ? 1.0f : ((q < 0) ? -1.0f : 0.0f);
    return __float2int_rz(floorf(q + 0.5f * sg));
}

// virtualVoxelPosToSDFBlock (RayCastRender.cu:28-33): (v < 0 ? v - 7 : v) / 8
// in C division is floor(v / 8), an arithmetic shift
static __device__ __forceinline__ int vox_to_block(int v) { return v >> 3; }

// virtualVoxelPosToLocal (RayCastRender.cu:36-42): ((v % 8) + 8) % 8 == v & 7
static __device__ __forceinline__ int vox_local(int v) { return v & 7; }

// Correctly rounded x / v for the fixed divisor v, given y = RN(1/v): one
// Markstein correction of the product x*y (P. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990): r = x - q v is exact and q + r y rounds to x / v.
// Used only for 2^-100 <= |x| < kDivRange, and only when k_verify_div found
// it equal to IEEE division for every float of that range with this v
// (checked at scene creation); near zero the product underflows and the
// correction is not exact, so those x use IEEE division.
constexpr float kDivRange = 1024.0f;
constexpr float kDivTiny = 0x1p-100f;
static __device__ __forceinline__ float div_fixed(float x, float v, float y) {
    const float q = __fmul_rn(x, y);
    const float r = __fmaf_rn(-q, v, x);
    return __fmaf_rn(r, y, q);
}

static __device__ __forceinline__ float div_v(float x, float v, float y, bool fast) {
    const float ax = fabsf(x);
    if (fast && ax >= kDivTiny && ax < kDivRange) return div_fixed(x, v, y);
    return x / v;
}

// getVoxel's block search (RayCastRender.cu:55-121) for the taps' blocks;
// -1 = block not allocated (the tap reads as weight 0).
static __device__ __forceinline__ void refill_taps(const SceneDev& s, TapCache& tc, int bx0, int by0, int bz0, int span,
                                            uint8_t* touched) {
    tc.bx = bx0;
    tc.by = by0;
    tc.bz = bz0;
    tc.span = span;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int c = i & span;
        if (c == i) {
            const int bx = bx0 + (i & 1), by = by0 + ((i >> 1) & 1), bz = bz0 + ((i >> 2) & 1);
            const int p = block_ptr(s, bx, by, bz);
            if (touched && p >= 0) touched[p] = 1;
            tc.set(i, p);
        } else {
            int p = tc.t0;
#pragma unroll
            for (int j = 1; j < i; ++j)
                if (c == j) p = tc.get(j);
            tc.set(i, p);
        }
    }
}

static __device__ __forceinline__ float frac01(float v) { return v - floorf(v); }


// Ray parameter interval inside the axis-aligned cell [c*S, (c+1)*S)^3.
// Approximate arithmetic: callers keep a margin from both ends.
struct RayInv {
    float ox, oy, oz, ix, iy, iz;
    bool hx, hy, hz;
};

static __device__ __forceinline__ void cell_interval(const RayInv& R, int cx, int cy, int cz, float S, float& tlo,
                                              float& thi) {
    tlo = -3.4e38f;
    thi = 3.4e38f;
    if (R.hx) {
        const float t0 = ((float)cx * S - R.ox) * R.ix, t1 = ((float)(cx + 1) * S - R.ox) * R.ix;
        tlo = fmaxf(tlo, fminf(t0, t1));
        thi = fminf(thi, fmaxf(t0, t1));
    }
    if (R.hy) {
        const float t0 = ((float)cy * S - R.oy) * R.iy, t1 = ((float)(cy + 1) * S - R.oy) * R.iy;
        tlo = fmaxf(tlo, fminf(t0, t1));
        thi = fminf(thi, fmaxf(t0, t1));
    }
    if (R.hz) {
        const float t0 = ((float)cz * S - R.oz) * R.iz, t1 = ((float)(cz + 1) * S - R.oz) * R.iz;
        tlo = fmaxf(tlo, fminf(t0, t1));
        thi = fminf(thi, fmaxf(t0, t1));
    }
}

// trilinearInterpolationSimpleFastFast, RayCastRender.cu:127-215.  The
// colour is only accumulated when asked for (it never steers the march).
static __device__ __forceinline__ bool trilinear(const SceneDev& s, float px, float py, float pz, float& dist,
                                          bool want_color, uint32_t& rgb, TapCache& tc, uint8_t* touched) {
    const float off = s.voxel;
    const float v = s.voxel;
    const float dx = px - off / 2.0f, dy = py - off / 2.0f, dz = pz - off / 2.0f;
    const bool fast = s.div_fast;
    const float y = s.inv_voxel;
    const float fx = div_v(dx, v, y, fast), fy = div_v(dy, v, y, fast), fz = div_v(dz, v, y, fast);
    const float wx = frac01(fx), wy = frac01(fy), wz = frac01(fz);
    const int ax0 = tap_voxel(fx), ay0 = tap_voxel(fy), az0 = tap_voxel(fz);
    const int ax1 = tap_voxel(div_v(dx + off, v, y, fast)), ay1 = tap_voxel(div_v(dy + off, v, y, fast)),
              az1 = tap_voxel(div_v(dz + off, v, y, fast));
    const int bx0 = vox_to_block(ax0), by0 = vox_to_block(ay0), bz0 = vox_to_block(az0);
    const int span = (vox_to_block(ax1) != bx0 ? 1 : 0) | (vox_to_block(ay1) != by0 ? 2 : 0) |
                     (vox_to_block(az1) != bz0 ? 4 : 0);
    if (!(tc.bx == bx0 && tc.by == by0 && tc.bz == bz0 && tc.span == span)) refill_taps(s, tc, bx0, by0, bz0, span, touched);
    const int lx0 = vox_local(ax0), ly0 = vox_local(ay0) * kBlock, lz0 = vox_local(az0) * kBlock * kBlock;
    const int lx1 = vox_local(ax1), ly1 = vox_local(ay1) * kBlock, lz1 = vox_local(az1) * kBlock * kBlock;
    uint2 raw[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        raw[i] = make_uint2(0u, 0u);
        if (tc.get(i) >= 0) {
            const int li = ((i & 1) ? lx1 : lx0) + ((i & 2) ? ly1 : ly0) + ((i & 4) ? lz1 : lz0);
            raw[i] = __ldg(reinterpret_cast<const uint2*>(s.voxels + (size_t)tc.get(i) * kVoxPerBlock + li));
        }
    }
    float d = 0.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f, vws = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if ((raw[i].y >> 24) == 0u) continue;
        const float w = ((i & 1) ? wx : (1.0f - wx)) * ((i & 2) ? wy : (1.0f - wy)) * ((i & 4) ? wz : (1.0f - wz));
        d += w * __uint_as_float(raw[i].x);
        if (want_color) {
            cr += w * (float)(raw[i].y & 0xFFu);
            cg += w * (float)((raw[i].y >> 8) & 0xFFu);
            cb += w * (float)((raw[i].y >> 16) & 0xFFu);
        }
        vws += w;
    }
    if (vws <= 1e-6f) return false;
    const float inv = 1.0f / vws;
    dist = d * inv;
    if (want_color) {
        cr *= inv;
        cg *= inv;
        cb *= inv;
        rgb = (uint32_t)(unsigned char)cr | ((uint32_t)(unsigned char)cg << 8) | ((uint32_t)(unsigned char)cb << 16);
    }
    return true;
}

// One ray: pixel (x, y) of the scene in a (in the image).  Warps should
// cover 8x4 pixel tiles of one scene.
static __device__ __forceinline__ void render_pixel(const RenderArgs& a, int x, int y) {
    const SceneDev& s = a.s;
    // numActiveBlocks == 0 leaves the outputs untouched (RayCastRender.cu:552-555)
    if (*(volatile int*)&s.ctr->free_count >= s.num_blocks) return;
    float T[12];
    if (a.pose_dev) {
#pragma unroll
        for (int i = 0; i < 12; ++i) T[i] = __ldg(a.pose_dev + i);
    } else {
#pragma unroll
        for (int i = 0; i < 12; ++i) T[i] = a.pose.T[i];
    }
    const size_t pi = (size_t)y * a.W + x;
    // renderKernel, RayCastRender.cu:447-500
    float cdx = ((float)x - a.cx) / a.fx, cdy = ((float)y - a.cy) / a.fy, cdz = 1.0f;
    const float cl = sqrtf(cdx * cdx + cdy * cdy + cdz * cdz);
    if (cl > 1e-6f) {
        cdx /= cl;
        cdy /= cl;
        cdz /= cl;
    }
    float wdx = T[0] * cdx + T[1] * cdy + T[2] * cdz;
    float wdy = T[4] * cdx + T[5] * cdy + T[6] * cdz;
    float wdz = T[8] * cdx + T[9] * cdy + T[10] * cdz;
    const float wl = sqrtf(wdx * wdx + wdy * wdy + wdz * wdz);
    if (wl > 1e-6f) {
        wdx /= wl;
        wdy /= wl;
        wdz /= wl;
    }
    float out_depth = kMinf;
    float4 out_pos = make_float4(kMinf, kMinf, kMinf, kMinf);
    float4 out_col = make_float4(kMinf, kMinf, kMinf, kMinf);
    bool hit = false;
    const float minD = a.minD, maxD = a.maxD;
    if (!(minD == 0 || minD == kMinf) && !(maxD == 0 || maxD == kMinf)) {
        // traverseCoarseGridSimpleSampleAll, RayCastRender.cu:276-398
        const float ox = a.camx, oy = a.camy, oz = a.camz;
        const float v = s.voxel;
        float lastSdf = 0.0f, lastAlpha = 0.0f;
        bool lastValid = false;
        const float d2r = 1.0f / cdz;
        float rc = d2r * fmaxf(minD, minD);
        const float re = d2r * fminf(maxD, maxD);
        const float C = (float)kBlock * v, C2 = 2.0f * v, C8 = 64.0f * v;
        const float invC2 = 1.0f / C2;
        RayInv R;
        R.ox = ox;
        R.oy = oy;
        R.oz = oz;
        R.hx = fabsf(wdx) > 1e-12f;
        R.hy = fabsf(wdy) > 1e-12f;
        R.hz = fabsf(wdz) > 1e-12f;
        R.ix = R.hx ? 1.0f / wdx : 0.0f;
        R.iy = R.hy ? 1.0f / wdy : 0.0f;
        R.iz = R.hz ? 1.0f / wdz : 0.0f;
        TapCache tc;
        tc.bx = 0x7FFFFFFF;
        tc.by = tc.bz = tc.span = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) tc.set(i, -1);
        int steps = 0;  // FP32 chain additions so far (iteration guard)
        uint32_t n_full = 0u, n_skip = 0u, n_jump = 0u, n_single = 0u;
        const float m = 1e-4f;  // keep skipped samples this far inside their cell
        // one loop for the march and the regula-falsi steps, so a single
        // trilinear evaluation site serves both (mode 0 = march, 1..3 =
        // step k of findIntersectionBisection, RayCastRender.cu:229-271)
        int mode = 0;
        float ba = 0.0f, bad = 0.0f, bb = 0.0f, bbd = 0.0f, bc = 0.0f, mdist = 0.0f;
        uint32_t rgb = 0u;
#pragma unroll 1
        while (true) {
            float st;  // ray parameter of the sample to evaluate
            if (mode == 0) {
                if (!(rc < re)) break;
                if (steps >= kMaxMarch) {
                    atomicOr(&s.ctr->flags, (uint32_t)VSG_FLAG_MARCH_LIMIT);
                    break;
                }
                const float spx = ox + rc * wdx, spy = oy + rc * wdy, spz = oz + rc * wdz;
                // global sub-cube (2 voxels) of the sample, its block cell and super-cell
                const int qx = __float2int_rd(spx * invC2), qy = __float2int_rd(spy * invC2),
                          qz = __float2int_rd(spz * invC2);
                float tlo = 0.0f, thi = 0.0f;
                bool cell = false;
                const int k = s.bidx_log2;
                const uint32_t sb = grid_bit(qx >> 5, qy >> 5, qz >> 5, k - 3);
                if (!((__ldg(s.sup + (sb >> 5)) >> (sb & 31)) & 1u)) {
                    cell_interval(R, qx >> 5, qy >> 5, qz >> 5, C8, tlo, thi);  // 64-voxel cell
                    cell = true;
                } else {
                    const unsigned long long w = __ldg(s.dwm + bidx_cell(qx >> 2, qy >> 2, qz >> 2, k));
                    if (w == 0ull) {
                        cell_interval(R, qx >> 2, qy >> 2, qz >> 2, C, tlo, thi);  // 8-voxel cell
                        cell = true;
                    } else if (!((w >> ((((qz & 3) << 2) | (qy & 3)) << 2 | (qx & 3))) & 1ull)) {
                        cell_interval(R, qx, qy, qz, C2, tlo, thi);  // 2-voxel cell
                        cell = true;
                    }
                }
                if (cell) {
                    if (rc > tlo + m && rc < thi - m) {
                        const int before = steps;
                        rc = vsg_chain_advance(rc, v * 0.5f, fminf(thi - m, re), kMaxMarch - steps, &steps);
                        n_skip += (uint32_t)(steps - before);
                        ++n_jump;
                        lastValid = false;
                        continue;
                    }
                    ++n_single;  // too close to the cell boundary to trust the test
                }
                st = rc;
            } else {
                st = bc;
            }
            float dist = 0.0f;
            ++n_full;
            const bool ok = trilinear(s, ox + st * wdx, oy + st * wdy, oz + st * wdz, dist, mode != 0, rgb, tc, a.touched);
            if (mode == 0) {
                if (ok && lastValid && lastSdf < 0.0f && dist > 0.0f) {
                    // zero crossing: a = last sample, b = this one
                    if (a.rec) a.rec[pi] = make_float2(lastAlpha, rc);
                    ba = lastAlpha;
                    bad = lastSdf;
                    bb = rc;
                    bbd = dist;
                    mdist = dist;
                    bc = ba + (bad / (bad - bbd)) * (bb - ba);  // findIntersectionLinear
                    mode = 1;
                    continue;
                }
                if (ok) {
                    lastSdf = dist;
                    lastAlpha = rc;
                }
                lastValid = ok;
                rc += v * 0.5f;
                ++steps;
            } else {
                bool finished = !ok, success = false;
                if (ok) {
                    if (bad * dist > 0.0f) {
                        ba = bc;
                        bad = dist;
                    } else {
                        bb = bc;
                        bbd = dist;
                    }
                    if (mode == 3) {
                        finished = true;
                        success = true;
                    } else {
                        bc = ba + (bad / (bad - bbd)) * (bb - ba);
                        ++mode;
                    }
                }
                if (finished) {
                    const float th = v * 3;  // RayCastRender.cu:362-365
                    if (success && fabsf(lastSdf - mdist) < th && fabsf(mdist) < th) {
                        const float alpha = bc;
                        out_depth = alpha / d2r;
                        out_pos = make_float4(ox + alpha * wdx, oy + alpha * wdy, oz + alpha * wdz, 1.0f);
                        out_col = make_float4((float)(rgb & 0xFFu) / 255.0f, (float)((rgb >> 8) & 0xFFu) / 255.0f,
                                              (float)((rgb >> 16) & 0xFFu) / 255.0f, 1.0f);
                        hit = true;
                        break;
                    }
                    // not accepted: the march continues after the crossing sample
                    lastSdf = mdist;
                    lastAlpha = rc;
                    lastValid = true;
                    rc += v * 0.5f;
                    ++steps;
                    mode = 0;
                }
            }
        }
        const unsigned am = __activemask();
        const unsigned hm = __ballot_sync(am, hit);
        const uint32_t it = n_full + n_jump;
        const uint32_t it_max = __reduce_max_sync(am, it);
        uint32_t nf = n_full, ns = n_skip, nj = n_jump, n1 = n_single, ni = it;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            nf += __shfl_xor_sync(am, nf, o);
            ns += __shfl_xor_sync(am, ns, o);
            nj += __shfl_xor_sync(am, nj, o);
            n1 += __shfl_xor_sync(am, n1, o);
            ni += __shfl_xor_sync(am, ni, o);
        }
        if ((threadIdx.x & 31) == (__ffs(am) - 1)) {
            atomicAdd(&s.frame->hits, (uint32_t)__popc(hm));
            atomicAdd(&s.frame->misses, (uint32_t)(__popc(am) - __popc(hm)));
            atomicAdd(&s.frame->samples_full, nf);
            atomicAdd(&s.frame->samples_skipped, ns);
            atomicAdd(&s.frame->jumps, nj);
            atomicAdd(&s.frame->singles, n1);
            atomicAdd(&s.frame->lane_iters, ni);
            atomicAdd(&s.frame->warp_iters, it_max);
        }
    }
    a.depth[pi] = out_depth;
    a.pos[pi] = out_pos;
    a.col[pi] = out_col;
    a.nrm[pi] = make_float4(kMinf, kMinf, kMinf, kMinf);
}

static __device__ __forceinline__ void render_begin(FrameCounters* f) {
    f->hits = 0u;
    f->misses = 0u;
    f->samples_full = 0u;
    f->samples_skipped = 0u;
    f->jumps = 0u;
    f->singles = 0u;
    f->blocks_read = 0u;
    f->lane_iters = 0u;
    f->warp_iters = 0u;
}

}  // namespace vsg
