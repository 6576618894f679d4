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
    // march step (metres); 0: the reference's half voxel (RayCastRender.cu:
    // 389-392).  Any other value is an opt-in approximation, not the drop-in.
    float step;
    float* depth;
    float4* pos;
    float4* col;
    float4* nrm;
    float2* rec;  // non-null when recording: per pixel the march bracket of its last zero crossing
    // Optional ray-distance bounds (k_tile_bounds): per 8x4 pixel tile, then
    // per 64x32 pixel tile, then one entry for every pixel; .x = ~bits of the
    // nearest, .y = bits of the farthest distance (0 / 0: no box).
    const uint2* bounds;
    int t1x, t2x, n1, n2;
};

// Pool indices of the blocks holding a sample's 8 trilinear taps.  The taps
// of one sample span at most two blocks per axis (tap voxels x0 <= x1 <=
// x0 + 2); tp[i] is the block of tap i.  Consecutive samples mostly reuse
// the same blocks, so the entry is kept across samples.  Unallocated blocks
// are entered as the pool's zero block (index num_blocks).
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

// lookup_block for the ray caster, out of line: the dense block index
// resolves almost every tap block, and keeping the rare bucket search out of
// the march loop keeps the loop's code small.
static __device__ __noinline__ int lookup_far(const Entry* buckets, const int* bucket_next, const Node* nodes,
                                              uint32_t nb, int max_nodes, int x, int y, int z) {
    const unsigned long long key = pack_key(x, y, z);
    const uint32_t b = bucket_of(x, y, z, nb);
    const Entry* bk = buckets + (size_t)b * kBucketSlots;
#pragma unroll
    for (int j = 0; j < kBucketSlots; ++j) {
        const uint4 e = __ldg(reinterpret_cast<const uint4*>(bk + j));
        const unsigned long long k = ((unsigned long long)e.y << 32) | e.x;
        if (k == key) return (int)e.z;
        if (k == kKeyEmpty) return -1;
    }
    int n = __ldg(bucket_next + b);
    for (int it = 0; n >= 0 && it < max_nodes; ++it) {
        const uint4 e = __ldg(reinterpret_cast<const uint4*>(nodes + n));
        const unsigned long long k = ((unsigned long long)e.y << 32) | e.x;
        if (k == key) return (int)e.z;
        n = (int)e.w;
    }
    return -1;
}

// block_ptr with the bucket search out of line
static __device__ __forceinline__ int block_ptr_r(const SceneDev& s, int x, int y, int z) {
    if (!coord_ok(x, y, z)) return -1;
    const unsigned long long e = __ldg(s.bindex + bidx_cell(x, y, z, s.bidx_log2));
    if (e == kIdxEmpty) return -1;
    if (e == kIdxShared) return lookup_far(s.buckets, s.bucket_next, s.nodes, s.num_buckets, s.max_nodes, x, y, z);
    return ((e >> 22) == bidx_tag(x, y, z, s.bidx_log2)) ? (int)(e & kIdxPtrMask) : -1;
}

// getVoxel's block search (RayCastRender.cu:55-121) for the taps' blocks; a
// block that is not allocated is entered as num_blocks, the all-zero block
// past the pool (its taps read as weight 0).
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
            const int p = block_ptr_r(s, bx, by, bz);
            if (touched && p >= 0) touched[p] = 1;
            tc.set(i, p >= 0 ? p : s.num_blocks);  // the zero block past the pool
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
    // the six quotients (sample and sample + one voxel, per axis) take the
    // verified fixed-divisor path together when all six dividends are in its
    // range (one test instead of six divergent ones), else one by one
    const float ex = dx + off, ey = dy + off, ez = dz + off;
    const float mn = fminf(fminf(fminf(fabsf(dx), fabsf(dy)), fminf(fabsf(dz), fabsf(ex))), fminf(fabsf(ey), fabsf(ez)));
    const float mx = fmaxf(fmaxf(fmaxf(fabsf(dx), fabsf(dy)), fmaxf(fabsf(dz), fabsf(ex))), fmaxf(fabsf(ey), fabsf(ez)));
    float fx, fy, fz, gx, gy, gz;
    if (fast && mn >= kDivTiny && mx < kDivRange) {
        fx = div_fixed(dx, v, y);
        fy = div_fixed(dy, v, y);
        fz = div_fixed(dz, v, y);
        gx = div_fixed(ex, v, y);
        gy = div_fixed(ey, v, y);
        gz = div_fixed(ez, v, y);
    } else {
        fx = div_v(dx, v, y, fast);
        fy = div_v(dy, v, y, fast);
        fz = div_v(dz, v, y, fast);
        gx = div_v(ex, v, y, fast);
        gy = div_v(ey, v, y, fast);
        gz = div_v(ez, v, y, fast);
    }
    const float wx = frac01(fx), wy = frac01(fy), wz = frac01(fz);
    const int ax0 = tap_voxel(fx), ay0 = tap_voxel(fy), az0 = tap_voxel(fz);
    const int ax1 = tap_voxel(gx), ay1 = tap_voxel(gy), az1 = tap_voxel(gz);
    const int bx0 = vox_to_block(ax0), by0 = vox_to_block(ay0), bz0 = vox_to_block(az0);
    const int span = (vox_to_block(ax1) != bx0 ? 1 : 0) | (vox_to_block(ay1) != by0 ? 2 : 0) |
                     (vox_to_block(az1) != bz0 ? 4 : 0);
    if (!(tc.bx == bx0 && tc.by == by0 && tc.bz == bz0 && tc.span == span)) refill_taps(s, tc, bx0, by0, bz0, span, touched);
    const int lx0 = vox_local(ax0), ly0 = vox_local(ay0) * kBlock, lz0 = vox_local(az0) * kBlock * kBlock;
    const int lx1 = vox_local(ax1), ly1 = vox_local(ay1) * kBlock, lz1 = vox_local(az1) * kBlock * kBlock;
    uint2 raw[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        {  // an unallocated tap block reads the pool's zero block (weight 0)
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

// The march state of one ray (traverseCoarseGridSimpleSampleAll,
// RayCastRender.cu:276-398, with the refinement of
// findIntersectionBisection, :229-271, run as modes 1..3 of the same loop).
struct RayState {
    RayInv R;          // origin (the camera) and inverse direction
    float wdx, wdy, wdz;
    float d2r, rc, re;
    float h;           // march step
    float lastSdf, lastAlpha;
    float ba, bad, bb, bbd, bc, mdist;
    TapCache tc;
    int steps;         // FP32 chain additions so far (iteration guard)
    int mode;          // 0 = march, 1..3 = regula-falsi step
    bool lastValid;
    uint32_t rgb;
    uint32_t n_full, n_skip, n_jump, n_single;
    float out_depth;
    float4 out_pos, out_col;
    bool hit;
};

// Does the launch march at all?  minDepth / maxDepth of 0 or MINF leave
// every output at MINF (renderKernel, RayCastRender.cu:463-470).
static __device__ __forceinline__ bool march_enabled(const RenderArgs& a) {
    return !(a.minD == 0 || a.minD == kMinf) && !(a.maxD == 0 || a.maxD == kMinf);
}

static __device__ __forceinline__ void load_pose(const RenderArgs& a, float T[12]) {
    if (a.pose_dev) {
#pragma unroll
        for (int i = 0; i < 12; ++i) T[i] = __ldg(a.pose_dev + i);
    } else {
#pragma unroll
        for (int i = 0; i < 12; ++i) T[i] = a.pose.T[i];
    }
}

// renderKernel, RayCastRender.cu:447-500: the ray of pixel (x, y) and the
// start of its march.
static __device__ __forceinline__ void ray_setup(const RenderArgs& a, const float T[12], int x, int y, RayState& r) {
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
    r.wdx = wdx;
    r.wdy = wdy;
    r.wdz = wdz;
    r.out_depth = kMinf;
    r.out_pos = make_float4(kMinf, kMinf, kMinf, kMinf);
    r.out_col = make_float4(kMinf, kMinf, kMinf, kMinf);
    r.hit = false;
    r.lastSdf = 0.0f;
    r.lastAlpha = 0.0f;
    r.lastValid = false;
    r.h = a.step > 0.0f ? a.step : a.s.voxel * 0.5f;
    r.d2r = 1.0f / cdz;
    r.rc = r.d2r * fmaxf(a.minD, a.minD);
    r.re = r.d2r * fminf(a.maxD, a.maxD);
    r.R.ox = a.camx;
    r.R.oy = a.camy;
    r.R.oz = a.camz;
    r.R.hx = fabsf(wdx) > 1e-12f;
    r.R.hy = fabsf(wdy) > 1e-12f;
    r.R.hz = fabsf(wdz) > 1e-12f;
    r.R.ix = r.R.hx ? 1.0f / wdx : 0.0f;
    r.R.iy = r.R.hy ? 1.0f / wdy : 0.0f;
    r.R.iz = r.R.hz ? 1.0f / wdz : 0.0f;
    r.tc.bx = 0x7FFFFFFF;
    r.tc.by = r.tc.bz = r.tc.span = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.tc.set(i, -1);
    r.steps = 0;
    r.mode = 0;
    r.ba = r.bad = r.bb = r.bbd = r.bc = r.mdist = 0.0f;
    r.rgb = 0u;
    r.n_full = r.n_skip = r.n_jump = r.n_single = 0u;
}

// Start the march at the nearest and end it after the farthest ray distance
// at which a sample of this pixel's tile can read a weighted voxel: every
// sample outside that range is invalid, so skipping it (the chain replayed
// exactly) or not taking it leaves the outputs as they are.  The margin
// covers the rounding of the sample position cam + rc * dir.
template <bool kCountSkips>
static __device__ __forceinline__ void apply_bounds(const RenderArgs& a, int x, int y, RayState& r) {
    const uint2 b1 = __ldg(a.bounds + (y >> 2) * a.t1x + (x >> 3));
    const uint2 b2 = __ldg(a.bounds + a.n1 + (y >> 5) * a.t2x + (x >> 6));
    const uint2 bg = __ldg(a.bounds + a.n1 + a.n2);
    const uint32_t lo_inv = max(max(b1.x, b2.x), bg.x), hi_bits = max(max(b1.y, b2.y), bg.y);
    if (lo_inv == 0u) {  // no weighted block projects onto the tile
        r.re = r.rc;
        return;
    }
    const float lo = __uint_as_float(~lo_inv), hi = __uint_as_float(hi_bits);
    const float cm = fmaxf(fmaxf(fabsf(r.R.ox), fabsf(r.R.oy)), fabsf(r.R.oz));
    const float first = lo - (1e-4f + 1e-4f * lo + 1e-6f * (cm + lo));
    const float last = hi + (1e-4f + 1e-4f * hi + 1e-6f * (cm + hi));
    r.re = fminf(r.re, last);
    if (first > r.rc && r.rc < r.re) {
        const int before = r.steps;
        r.rc = vsg_chain_advance(r.rc, r.h, fminf(first, r.re), kMaxMarch - r.steps, &r.steps);
        if (kCountSkips) r.n_skip += (uint32_t)(r.steps - before);
        ++r.n_jump;
    }
}

// Ray-distance bounds per pixel tile for the march (apply_bounds).  One
// thread per pool block.  A block that holds a weighted voxel (or has not
// been integrated yet: all of it) is taken as the bounding box of its
// weighted 2x2x2 sub-cubes grown by 2 voxels: the taps of a sample at p are
// voxels floor(p/v) - 1 .. floor(p/v) + 1 per axis (RayCastRender.cu:17-25,
// 127-170, whose round-half-away-from-zero reaches one voxel lower for
// negative coordinates), so a sample can only read voxel i from within one
// voxel of it, and the second voxel of growth is slack.  The part of the box
// in front of the plane at half the minimum depth (every sample is at least
// the minimum depth ahead of the camera) is projected; its pixel rectangle,
// grown by a 2-pixel margin, is entered into the 8x4 tiles it covers (up to
// 64 of them), else into the 64x32 tiles (up to 4096), else into the entry
// for every pixel: nearest distance by atomicMax of ~bits, farthest by
// atomicMax of bits (non-negative floats order like their bits).  A pose
// whose rotation is not orthonormal, a zero focal length or a non-positive
// minimum depth disables the bounds (nearest 0, farthest infinity).
// Pool blocks first, first + stride, ... of one render's scene.
static __device__ __forceinline__ void tile_bounds_range(const RenderArgs& a, uint32_t first, uint32_t stride) {
    const SceneDev& s = a.s;
    unsigned* bnd = reinterpret_cast<unsigned*>(const_cast<uint2*>(a.bounds));
    unsigned* glob = bnd + 2 * (a.n1 + a.n2);
    float T[12];
    load_pose(a, T);
    float e = 0.0f;  // largest entry of R^T R - I
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float d = T[i] * T[j] + T[4 + i] * T[4 + j] + T[8 + i] * T[8 + j] - (i == j ? 1.0f : 0.0f);
            e = fmaxf(e, fabsf(d));
        }
    const bool ok = e < 1e-4f && isfinite(a.fx) && isfinite(a.fy) && a.fx != 0.0f && a.fy != 0.0f &&
                    isfinite(a.cx) && isfinite(a.cy) && a.minD > 0.0f && isfinite(a.minD) && isfinite(a.camx) &&
                    isfinite(a.camy) && isfinite(a.camz);
    if (!ok) {
        if (first == 0u) {
            atomicMax(glob, 0xFFFFFFFFu);  // nearest 0
            atomicMax(glob + 1, 0x7F800000u);  // farthest +inf
        }
        return;
    }
    const float zc = 0.5f * a.minD;
    const float mpx = 2.0f + 10.0f * e * (fabsf(a.fx) + fabsf(a.fy) + (float)a.W + (float)a.H);
    const float v = s.voxel;
    const uint32_t hw = s.ctr->high_water;
    for (uint32_t b = first; b < hw; b += stride) {
        const unsigned long long key = s.block_key[b];
        if (key == kKeyEmpty || key == kKeyTomb) continue;
        const unsigned long long wm = s.block_fresh[b] ? ~0ull : s.block_wmask[b];
        if (wm == 0ull) continue;
        int bx, by, bz;
        unpack_key(key, bx, by, bz);
        // occupied sub-cube rows per axis (bit (sz*4+sy)*4+sx of wm)
        unsigned long long f = wm | (wm >> 32);
        f |= f >> 16;
        const unsigned yz = (unsigned)(f & 0xFFFFull);  // (sy, sx) over all sz
        unsigned xm = yz | (yz >> 8);
        xm = (xm | (xm >> 4)) & 0xFu;
        const unsigned ym = ((yz & 0xFu) ? 1u : 0u) | ((yz & 0xF0u) ? 2u : 0u) | ((yz & 0xF00u) ? 4u : 0u) |
                            ((yz & 0xF000u) ? 8u : 0u);
        const unsigned zm = ((wm & 0xFFFFull) ? 1u : 0u) | ((wm & 0xFFFF0000ull) ? 2u : 0u) |
                            ((wm & 0xFFFF00000000ull) ? 4u : 0u) | ((wm & 0xFFFF000000000000ull) ? 8u : 0u);
        const int sx0 = __ffs(xm) - 1, sx1 = 31 - __clz(xm), sy0 = __ffs(ym) - 1, sy1 = 31 - __clz(ym);
        const int sz0 = __ffs(zm) - 1, sz1 = 31 - __clz(zm);
        const float lo[3] = {((float)(bx * kBlock + 2 * sx0) - 2.0f) * v, ((float)(by * kBlock + 2 * sy0) - 2.0f) * v,
                             ((float)(bz * kBlock + 2 * sz0) - 2.0f) * v};
        const float hi[3] = {((float)(bx * kBlock + 2 * sx1) + 4.0f) * v, ((float)(by * kBlock + 2 * sy1) + 4.0f) * v,
                             ((float)(bz * kBlock + 2 * sz1) + 4.0f) * v};
        const float c[3] = {a.camx, a.camy, a.camz};
        float n2 = 0.0f, f2 = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float dl = lo[i] - c[i], dh = hi[i] - c[i];
            const float n = fmaxf(fmaxf(dl, -dh), 0.0f), f = fmaxf(fabsf(dl), fabsf(dh));
            n2 += n * n;
            f2 += f * f;
        }
        const float dmin = sqrtf(n2), dmax = sqrtf(f2);
        // camera coordinates of the 8 corners
        float px[8], py[8], pz[8];
        bool any_front = false;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float dx = ((k & 1) ? hi[0] : lo[0]) - c[0];
            const float dy = ((k & 2) ? hi[1] : lo[1]) - c[1];
            const float dz = ((k & 4) ? hi[2] : lo[2]) - c[2];
            px[k] = T[0] * dx + T[4] * dy + T[8] * dz;
            py[k] = T[1] * dx + T[5] * dy + T[9] * dz;
            pz[k] = T[2] * dx + T[6] * dy + T[10] * dz;
            any_front |= pz[k] >= zc;
        }
        if (!any_front) continue;  // wholly nearer than any sample
        float u0 = 3.4e38f, u1 = -3.4e38f, w0 = 3.4e38f, w1 = -3.4e38f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (pz[k] >= zc) {
                const float u = a.fx * (px[k] / pz[k]) + a.cx, w = a.fy * (py[k] / pz[k]) + a.cy;
                u0 = fminf(u0, u);
                u1 = fmaxf(u1, u);
                w0 = fminf(w0, w);
                w1 = fmaxf(w1, w);
            }
        }
        // edges crossing the plane z = zc (corners k and k ^ axis bit)
#pragma unroll
        for (int k = 0; k < 8; ++k)
#pragma unroll
            for (int ax = 1; ax < 8; ax <<= 1) {
                if (k & ax) continue;
                const int j = k | ax;
                if ((pz[k] >= zc) == (pz[j] >= zc)) continue;
                const float t = (zc - pz[k]) / (pz[j] - pz[k]);
                const float qx = px[k] + t * (px[j] - px[k]), qy = py[k] + t * (py[j] - py[k]);
                const float u = a.fx * (qx / zc) + a.cx, w = a.fy * (qy / zc) + a.cy;
                u0 = fminf(u0, u);
                u1 = fmaxf(u1, u);
                w0 = fminf(w0, w);
                w1 = fmaxf(w1, w);
            }
        u0 -= mpx;
        u1 += mpx;
        w0 -= mpx;
        w1 += mpx;
        if (!(u1 >= 0.0f && w1 >= 0.0f && u0 <= (float)(a.W - 1) && w0 <= (float)(a.H - 1))) continue;
        const int x0 = (int)fmaxf(u0, 0.0f), x1 = (int)fminf(u1, (float)(a.W - 1));
        const int y0 = (int)fmaxf(w0, 0.0f), y1 = (int)fminf(w1, (float)(a.H - 1));
        const unsigned lo_inv = ~__float_as_uint(dmin), hi_bits = __float_as_uint(dmax);
        const int ax0 = x0 >> 3, ax1 = x1 >> 3, ay0 = y0 >> 2, ay1 = y1 >> 2;
        if ((ax1 - ax0 + 1) * (ay1 - ay0 + 1) <= 64) {
            for (int ty = ay0; ty <= ay1; ++ty)
                for (int tx = ax0; tx <= ax1; ++tx) {
                    unsigned* e1 = bnd + 2 * (ty * a.t1x + tx);
                    atomicMax(e1, lo_inv);
                    atomicMax(e1 + 1, hi_bits);
                }
            continue;
        }
        const int bx0 = x0 >> 6, bx1 = x1 >> 6, by0 = y0 >> 5, by1 = y1 >> 5;
        if ((bx1 - bx0 + 1) * (by1 - by0 + 1) <= 4096) {
            for (int ty = by0; ty <= by1; ++ty)
                for (int tx = bx0; tx <= bx1; ++tx) {
                    unsigned* e2 = bnd + 2 * (a.n1 + ty * a.t2x + tx);
                    atomicMax(e2, lo_inv);
                    atomicMax(e2 + 1, hi_bits);
                }
            continue;
        }
        atomicMax(glob, lo_inv);
        atomicMax(glob + 1, hi_bits);
    }
}

// Ray-cast tile order, longest march first.  A CTA tile of 16x8 pixels
// holds four 8x4 bound tiles; its weight is the largest distance range
// [nearest, farthest] its rays may march (apply_bounds), bucketed by powers
// of two of march steps.  The tiles with the longest ranges are cast first,
// so the last wave of the launch holds short ones instead of a long tail.
// Each pixel's result does not depend on the order.
constexpr int kOrderBuckets = 16;

static __device__ __forceinline__ int tile_bucket(const RenderArgs& a, int tx, int ty) {
    const int t1y = a.n1 / a.t1x;
    const uint2 bg = __ldg(a.bounds + a.n1 + a.n2);
    float cost = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int x8 = 2 * tx + (k & 1), y4 = 2 * ty + (k >> 1);
        if (x8 >= a.t1x || y4 >= t1y) continue;
        const uint2 b1 = __ldg(a.bounds + y4 * a.t1x + x8);
        const uint2 b2 = __ldg(a.bounds + a.n1 + (y4 >> 3) * a.t2x + (x8 >> 3));
        const uint32_t lo_inv = max(max(b1.x, b2.x), bg.x), hi_bits = max(max(b1.y, b2.y), bg.y);
        if (lo_inv == 0u) continue;
        cost = fmaxf(cost, __uint_as_float(hi_bits) - __uint_as_float(~lo_inv));
    }
    if (!(cost > 0.0f)) return 0;
    const float steps = cost / (0.5f * a.s.voxel);
    if (!(steps < 3.0e38f)) return kOrderBuckets - 1;
    const int e = (int)((__float_as_uint(fmaxf(steps, 1.0f)) >> 23) & 0xFFu) - 127;  // floor(log2(steps))
    return 1 + min(max(e, 0), kOrderBuckets - 2);
}

// One iteration of the march: a skip jump, a march sample or a
// regula-falsi sample.  Returns true when the ray is done.
template <bool kCountSkips>
static __device__ __forceinline__ bool ray_step(const RenderArgs& a, RayState& r, size_t pi) {
    const SceneDev& s = a.s;
    const float v = s.voxel;
    const float ox = r.R.ox, oy = r.R.oy, oz = r.R.oz;
    float st;  // ray parameter of the sample to evaluate
    if (r.mode == 0) {
        if (!(r.rc < r.re)) return true;
        if (r.steps >= kMaxMarch) {
            atomicOr(&s.ctr->flags, (uint32_t)VSG_FLAG_MARCH_LIMIT);
            return true;
        }
        const float C = (float)kBlock * v, C2 = 2.0f * v, C8 = 64.0f * v;
        // RN(1 / (2 v)) = RN(1 / v) / 2 exactly (halving a normal float is exact);
        // the batched caster reads the voxel size from memory, where the
        // division would not leave the loop
        const float invC2 = 0.5f * s.inv_voxel;
        const float m = 1e-4f;  // keep skipped samples this far inside their cell
        const float spx = ox + r.rc * r.wdx, spy = oy + r.rc * r.wdy, spz = oz + r.rc * r.wdz;
        // global sub-cube (2 voxels) of the sample, its block cell and super-cell
        const int qx = __float2int_rd(spx * invC2), qy = __float2int_rd(spy * invC2), qz = __float2int_rd(spz * invC2);
        float tlo = 0.0f, thi = 0.0f;
        bool cell = false;
        const int k = s.bidx_log2;
        const uint32_t sb = grid_bit(qx >> 5, qy >> 5, qz >> 5, k - 3);
        // Both grid words are loaded together (the dwm word is read even when
        // the super-cell is empty; every index is inside the grid), and the
        // empty cell, if any, goes through one cell_interval for all three
        // sizes, so lanes at different levels do not run separate copies.
        int sh = -1;  // the empty cell: 64-voxel (5), 8-voxel (2), 2-voxel (0), none (-1)
        const uint32_t supw = __ldg(s.sup + (sb >> 5));
        const unsigned long long w = __ldg(s.dwm + bidx_cell(qx >> 2, qy >> 2, qz >> 2, k));
        if (!((supw >> (sb & 31)) & 1u)) {
            sh = 5;
        } else if (w == 0ull) {
            sh = 2;
        } else {
            if (!((w >> ((((qz & 3) << 2) | (qy & 3)) << 2 | (qx & 3))) & 1ull))
                sh = 0;
        }
        if (sh >= 0) {
            cell_interval(r.R, qx >> sh, qy >> sh, qz >> sh, sh == 5 ? C8 : (sh == 2 ? C : C2), tlo, thi);
            cell = true;
        }
        if (cell) {
            if (r.rc > tlo + m && r.rc < thi - m) {
                // the march's own additions for a short skip (up to 8 steps,
                // exact by construction and cheaper than the O(1) replay),
                // vsg_chain_advance for the rest of a longer one
                const int before = r.steps;
                const float tgt = fminf(thi - m, r.re);
                float rc = r.rc;
                int n = 0;
#pragma unroll 1
                while (rc < tgt && n < 8 && r.steps + n < kMaxMarch) {
                    rc = rc + r.h;
                    ++n;
                }
                r.steps += n;
                if (rc < tgt) rc = vsg_chain_advance(rc, r.h, tgt, kMaxMarch - r.steps, &r.steps);
                r.rc = rc;
                if (kCountSkips) r.n_skip += (uint32_t)(r.steps - before);
                ++r.n_jump;
                r.lastValid = false;
                return false;
            }
            if (kCountSkips) ++r.n_single;  // too close to the cell boundary to trust the test
        }
        st = r.rc;
    } else {
        st = r.bc;
    }
    float dist = 0.0f;
    ++r.n_full;
    const bool ok = trilinear(s, ox + st * r.wdx, oy + st * r.wdy, oz + st * r.wdz, dist, r.mode != 0, r.rgb, r.tc,
                              a.touched);
    if (r.mode == 0) {
        if (ok && r.lastValid && r.lastSdf < 0.0f && dist > 0.0f) {
            // zero crossing: a = last sample, b = this one
            if (a.rec) a.rec[pi] = make_float2(r.lastAlpha, r.rc);
            r.ba = r.lastAlpha;
            r.bad = r.lastSdf;
            r.bb = r.rc;
            r.bbd = dist;
            r.mdist = dist;
            r.bc = r.ba + (r.bad / (r.bad - r.bbd)) * (r.bb - r.ba);  // findIntersectionLinear
            r.mode = 1;
            return false;
        }
        if (ok) {
            r.lastSdf = dist;
            r.lastAlpha = r.rc;
        }
        r.lastValid = ok;
        r.rc += r.h;
        ++r.steps;
        return false;
    }
    bool finished = !ok, success = false;
    if (ok) {
        if (r.bad * dist > 0.0f) {
            r.ba = r.bc;
            r.bad = dist;
        } else {
            r.bb = r.bc;
            r.bbd = dist;
        }
        if (r.mode == 3) {
            finished = true;
            success = true;
        } else {
            r.bc = r.ba + (r.bad / (r.bad - r.bbd)) * (r.bb - r.ba);
            ++r.mode;
        }
    }
    if (finished) {
        const float th = v * 3;  // RayCastRender.cu:362-365
        if (success && fabsf(r.lastSdf - r.mdist) < th && fabsf(r.mdist) < th) {
            const float alpha = r.bc;
            r.out_depth = alpha / r.d2r;
            r.out_pos = make_float4(ox + alpha * r.wdx, oy + alpha * r.wdy, oz + alpha * r.wdz, 1.0f);
            r.out_col = make_float4((float)(r.rgb & 0xFFu) / 255.0f, (float)((r.rgb >> 8) & 0xFFu) / 255.0f,
                                    (float)((r.rgb >> 16) & 0xFFu) / 255.0f, 1.0f);
            r.hit = true;
            return true;
        }
        // not accepted: the march continues after the crossing sample
        r.lastSdf = r.mdist;
        r.lastAlpha = r.rc;
        r.lastValid = true;
        r.rc += r.h;
        ++r.steps;
        r.mode = 0;
    }
    return false;
}

static __device__ __forceinline__ void ray_write(const RenderArgs& a, const RayState& r, size_t pi) {
    a.depth[pi] = r.out_depth;
    a.pos[pi] = r.out_pos;
    a.col[pi] = r.out_col;
    a.nrm[pi] = make_float4(kMinf, kMinf, kMinf, kMinf);
}

// Warp-summed march statistics of the active lanes into the frame counters.
static __device__ __forceinline__ void add_stats(const SceneDev& s, unsigned am, uint32_t hits, uint32_t rays,
                                                 uint32_t nf, uint32_t ns, uint32_t nj, uint32_t n1, uint32_t ni,
                                                 uint32_t witer) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        hits += __shfl_xor_sync(am, hits, o);
        rays += __shfl_xor_sync(am, rays, o);
        nf += __shfl_xor_sync(am, nf, o);
        ns += __shfl_xor_sync(am, ns, o);
        nj += __shfl_xor_sync(am, nj, o);
        n1 += __shfl_xor_sync(am, n1, o);
        ni += __shfl_xor_sync(am, ni, o);
    }
    if ((threadIdx.x & 31) == (__ffs(am) - 1)) {
        atomicAdd(&s.frame->hits, hits);
        atomicAdd(&s.frame->misses, rays - hits);
        atomicAdd(&s.frame->samples_full, nf);
        atomicAdd(&s.frame->samples_skipped, ns);
        atomicAdd(&s.frame->jumps, nj);
        atomicAdd(&s.frame->singles, n1);
        atomicAdd(&s.frame->lane_iters, ni);
        atomicAdd(&s.frame->warp_iters, witer);
    }
}

// One ray: pixel (x, y) of the scene in a (in the image).  Warps should
// cover 8x4 pixel tiles of one scene.  kCountSkips: also count the samples
// skipped as empty and the samples taken at a skip-cell boundary (the
// render_samples_skipped / render_singles statistics).  Those two counters
// cost about 10 % of the march (registers and instructions in the jump path
// of every iteration), so the kernels count them only in instrumented runs.
template <bool kCountSkips>
static __device__ __forceinline__ void render_pixel(const RenderArgs& a, int x, int y) {
    const SceneDev& s = a.s;
    // numActiveBlocks == 0 leaves the outputs untouched (RayCastRender.cu:552-555)
    if (*(volatile int*)&s.ctr->free_count >= s.num_blocks) return;
    float T[12];
    load_pose(a, T);
    const size_t pi = (size_t)y * a.W + x;
    RayState r;
    ray_setup(a, T, x, y, r);
    if (march_enabled(a)) {
        if (a.bounds) apply_bounds<kCountSkips>(a, x, y, r);
#pragma unroll 1
        while (!ray_step<kCountSkips>(a, r, pi)) {
        }
        const unsigned am = __activemask();
        const uint32_t it = r.n_full + r.n_jump;
        add_stats(s, am, r.hit ? 1u : 0u, 1u, r.n_full, r.n_skip, r.n_jump, r.n_single, it, __reduce_max_sync(am, it));
    }
    ray_write(a, r, pi);
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
