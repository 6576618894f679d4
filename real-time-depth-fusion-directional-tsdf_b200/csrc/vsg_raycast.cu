// vsg_raycast.cu -- ray caster (RayCastRender.cu:14-620 restated).
//
// One thread per pixel, warps on 8x4 pixel tiles.  The march replays the
// reference's fixed half-voxel FP32 step sequence exactly (rayCurrent +=
// 0.5 v, RayCastRender.cu:389-392) so hits, depths and colours match the
// reference bit for bit, but skips the work of samples that cannot be valid:
//   - block-cell DDA over the dilated occupancy grid: inside a cell whose
//     3x3x3 block neighbourhood holds no allocated block, every trilinear tap
//     of every sample misses, so the samples are invalid; only the FP32 step
//     additions are replayed;
//   - inside occupied cells, a tap in a block whose raw occupancy bit is
//     clear is a miss without a hash probe; the last probed block is cached.
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/vsg.h"
#include "vsg_device.cuh"
#include "vsg_internal.h"

namespace vsg {

constexpr int kMaxMarch = 1 << 22;  // iteration guard of one ray

struct RenderArgs {
    SceneDev s;
    int W, H;
    float camx, camy, camz;
    Pose pose;
    const float* pose_dev;
    float fx, fy, cx, cy, minD, maxD;
    float* depth;
    float4* pos;
    float4* col;
    float4* nrm;
};

struct TapCache {
    unsigned long long key;
    int ptr;
};

// worldToVirtualVoxelPos, RayCastRender.cu:17-25 (floorf variant)
__device__ __forceinline__ int tap_voxel(float q) {
    const float sg = (q > 0) ? 1.0f : ((q < 0) ? -1.0f : 0.0f);
    return __float2int_rz(floorf(q + 0.5f * sg));
}

__device__ __forceinline__ int vox_to_block(int v) {
    if (v < 0) v = (int)((unsigned)v - 7u);  // RayCastRender.cu:28-33
    return v / kBlock;
}

__device__ __forceinline__ int vox_local(int v) { return ((v % kBlock) + kBlock) % kBlock; }

// getVoxel, RayCastRender.cu:55-121: returns false for a missing block.
__device__ __forceinline__ bool fetch_voxel(const SceneDev& s, int vx, int vy, int vz, TapCache& tc,
                                            Voxel& out) {
    const int bx = vox_to_block(vx), by = vox_to_block(vy), bz = vox_to_block(vz);
    if (!occ_test(s.occ_raw, bx, by, bz, s.occ_log2)) return false;
    if (!coord_ok(bx, by, bz)) return false;
    const unsigned long long key = pack_key(bx, by, bz);
    if (key != tc.key) {
        tc.key = key;
        tc.ptr = lookup_block(s, key, bx, by, bz);
    }
    if (tc.ptr < 0) return false;
    const int li = vox_local(vx) + vox_local(vy) * kBlock + vox_local(vz) * kBlock * kBlock;
    const uint2 u = __ldg(reinterpret_cast<const uint2*>(s.voxels + (size_t)tc.ptr * kVoxPerBlock + li));
    out.sdf = __uint_as_float(u.x);
    out.rgbw = u.y;
    return true;
}

__device__ __forceinline__ float frac01(float v) { return v - floorf(v); }

// trilinearInterpolationSimpleFastFast, RayCastRender.cu:127-215.  The
// colour is only accumulated when asked for (it never steers the march).
__device__ __forceinline__ bool trilinear(const SceneDev& s, float px, float py, float pz, float& dist, bool want_color,
                          uint32_t& rgb, TapCache& tc) {
    const float off = s.voxel;
    const float v = s.voxel;
    const float dx = px - off / 2.0f, dy = py - off / 2.0f, dz = pz - off / 2.0f;
    const float fx = dx / v, fy = dy / v, fz = dz / v;
    const float wx = frac01(fx), wy = frac01(fy), wz = frac01(fz);
    const int ax0 = tap_voxel(fx), ay0 = tap_voxel(fy), az0 = tap_voxel(fz);
    const int ax1 = tap_voxel((dx + off) / v), ay1 = tap_voxel((dy + off) / v), az1 = tap_voxel((dz + off) / v);
    float d = 0.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f, vws = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        Voxel vx;
        if (!fetch_voxel(s, (i & 1) ? ax1 : ax0, (i & 2) ? ay1 : ay0, (i & 4) ? az1 : az0, tc, vx)) continue;
        if ((vx.rgbw >> 24) == 0u) continue;
        const float w = ((i & 1) ? wx : (1.0f - wx)) * ((i & 2) ? wy : (1.0f - wy)) * ((i & 4) ? wz : (1.0f - wz));
        d += w * vx.sdf;
        if (want_color) {
            cr += w * (float)(vx.rgbw & 0xFFu);
            cg += w * (float)((vx.rgbw >> 8) & 0xFFu);
            cb += w * (float)((vx.rgbw >> 16) & 0xFFu);
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

// findIntersectionBisection, RayCastRender.cu:229-271.
__device__ __forceinline__ bool bisection(const SceneDev& s, float ox, float oy, float oz, float wx, float wy, float wz, float d0,
                          float r0, float d1, float r1, float& alpha, uint32_t& rgb, TapCache& tc) {
    float a = r0, ad = d0, b = r1, bd = d1, c = 0.0f;
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        c = a + (ad / (ad - bd)) * (b - a);
        float cd;
        if (!trilinear(s, ox + c * wx, oy + c * wy, oz + c * wz, cd, true, rgb, tc)) return false;
        if (ad * cd > 0.0f) {
            a = c;
            ad = cd;
        } else {
            b = c;
            bd = cd;
        }
    }
    alpha = c;
    return true;
}

__global__ void __launch_bounds__(128) k_render(RenderArgs a) {
    const SceneDev& s = a.s;
    // numActiveBlocks == 0 leaves the outputs untouched (RayCastRender.cu:552-555)
    if (*(volatile int*)&s.ctr->free_count >= s.num_blocks) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    const int y = blockIdx.y * 8 + (warp >> 1) * 4 + (lane >> 3);
    if (x >= a.W || y >= a.H) return;
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
        const float h = v * 0.5f;
        const float C = (float)kBlock * v;
        const float invC = 1.0f / C;
        const bool hx = fabsf(wdx) > 1e-12f, hy = fabsf(wdy) > 1e-12f, hz = fabsf(wdz) > 1e-12f;
        const float ix = hx ? 1.0f / wdx : 0.0f, iy = hy ? 1.0f / wdy : 0.0f, iz = hz ? 1.0f / wdz : 0.0f;
        TapCache tc{kKeyEmpty, -1};
        int guard = 0;
#pragma unroll 1
        while (rc < re) {
            if (++guard > kMaxMarch) {
                atomicOr(&s.ctr->flags, (uint32_t)VSG_FLAG_MARCH_LIMIT);
                break;
            }
            const float spx = ox + rc * wdx, spy = oy + rc * wdy, spz = oz + rc * wdz;
            const int cx = __float2int_rd(spx * invC), cy = __float2int_rd(spy * invC),
                      cz = __float2int_rd(spz * invC);
            if (!occ_test(s.occ_dil, cx, cy, cz, s.occ_log2)) {
                // parameter interval of the ray inside cell (cx,cy,cz)
                float tlo = -3.4e38f, thi = 3.4e38f;
                if (hx) {
                    const float t0 = ((float)cx * C - ox) * ix, t1 = ((float)(cx + 1) * C - ox) * ix;
                    tlo = fmaxf(tlo, fminf(t0, t1));
                    thi = fminf(thi, fmaxf(t0, t1));
                }
                if (hy) {
                    const float t0 = ((float)cy * C - oy) * iy, t1 = ((float)(cy + 1) * C - oy) * iy;
                    tlo = fmaxf(tlo, fminf(t0, t1));
                    thi = fminf(thi, fmaxf(t0, t1));
                }
                if (hz) {
                    const float t0 = ((float)cz * C - oz) * iz, t1 = ((float)(cz + 1) * C - oz) * iz;
                    tlo = fmaxf(tlo, fminf(t0, t1));
                    thi = fminf(thi, fmaxf(t0, t1));
                }
                const float m = 1e-5f;
                const float tstop = fminf(thi - m, re);
                if (rc > tlo + m && rc < tstop) {
                    lastValid = false;
                    int n = 0;
#pragma unroll 1
                    do {
                        rc += h;
                    } while (rc < tstop && ++n < kMaxMarch);
                    continue;
                }
            }
            float dist;
            uint32_t rgb_unused = 0;
            if (trilinear(s, spx, spy, spz, dist, false, rgb_unused, tc)) {
                if (lastValid && lastSdf < 0.0f && dist > 0.0f) {
                    float alpha = 0.0f;
                    uint32_t rgb = 0;
                    const bool b = bisection(s, ox, oy, oz, wdx, wdy, wdz, lastSdf, lastAlpha, dist, rc, alpha, rgb, tc);
                    const float isx = ox + alpha * wdx, isy = oy + alpha * wdy, isz = oz + alpha * wdz;
                    const float th = v * 3;
                    if (b && fabsf(lastSdf - dist) < th) {
                        if (fabsf(dist) < th) {
                            out_depth = alpha / d2r;
                            out_pos = make_float4(isx, isy, isz, 1.0f);
                            out_col = make_float4((float)(rgb & 0xFFu) / 255.0f, (float)((rgb >> 8) & 0xFFu) / 255.0f,
                                                  (float)((rgb >> 16) & 0xFFu) / 255.0f, 1.0f);
                            hit = true;
                            break;
                        }
                    }
                }
                lastSdf = dist;
                lastAlpha = rc;
                lastValid = true;
                rc += v * 0.5f;
            } else {
                lastValid = false;
                rc += v * 0.5f;
            }
        }
        const unsigned hm = __ballot_sync(__activemask(), hit);
        const unsigned am = __activemask();
        if ((threadIdx.x & 31) == (__ffs(am) - 1)) {
            atomicAdd(&s.frame->hits, (uint32_t)__popc(hm));
            atomicAdd(&s.frame->misses, (uint32_t)(__popc(am) - __popc(hm)));
        }
    }
    a.depth[pi] = out_depth;
    a.pos[pi] = out_pos;
    a.col[pi] = out_col;
    a.nrm[pi] = make_float4(kMinf, kMinf, kMinf, kMinf);
}

__global__ void k_render_begin(FrameCounters* f) {
    f->hits = 0u;
    f->misses = 0u;
}

int render_launch(Renderer* r, Scene* sc, const float cam[3], const float* pose_dev, const float* pose_host,
                  float fx, float fy, float cx, float cy, float min_depth, float max_depth, cudaStream_t st) {
    RenderArgs a;
    a.s = sc->dev;
    a.W = r->w;
    a.H = r->h;
    a.camx = cam[0];
    a.camy = cam[1];
    a.camz = cam[2];
    if (pose_host)
        memcpy(a.pose.T, pose_host, sizeof(a.pose.T));
    else
        memset(a.pose.T, 0, sizeof(a.pose.T));
    a.pose_dev = pose_dev;
    a.fx = fx;
    a.fy = fy;
    a.cx = cx;
    a.cy = cy;
    a.minD = min_depth;
    a.maxD = max_depth;
    a.depth = r->depth;
    a.pos = r->position;
    a.col = r->color;
    a.nrm = r->normal;
    k_render_begin<<<1, 1, 0, st>>>(sc->dev.frame);
    dim3 grid((r->w + 15) / 16, (r->h + 7) / 8);
    timing_begin(sc, kSlotRender, st);
    k_render<<<grid, 128, 0, st>>>(a);
    timing_end(sc, kSlotRender, st);
    return cudaGetLastError() == cudaSuccess ? VSG_OK : VSG_ERR_CUDA;
}

}  // namespace vsg
