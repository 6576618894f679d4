// vsg_raycast.cu -- ray caster (RayCastRender.cu:14-620 restated).
//
// One thread per pixel, warps on 8x4 pixel tiles.  The march visits the
// reference's FP32 sample sequence exactly (rayCurrent += 0.5 v,
// RayCastRender.cu:389-392) so hits, depths and colours match the reference
// bit for bit, but only evaluates samples that can be valid:
// a sample's 8 taps lie in voxels floor(p/v)-1 .. floor(p/v)+2 per axis
// (RayCastRender.cu:17-25, 127-170, with a voxel of slack for rounding), so
// it can only be valid if a weighted voxel lies within one 2x2x2 sub-cube of
// the sample's sub-cube.  The dwm grid holds that bit per sub-cube (one
// 64-bit word per block position), the sup grid one bit per 8^3 block
// positions.  Cells whose bit is clear are skipped whole:
//   64-voxel cells (sup bit clear), 8-voxel cells (dwm word zero),
//   2-voxel cells (dwm bit clear).
// Skipped runs are replayed in O(1) by vsg_chain_advance, which lands on the
// exact float the serial additions produce.  Surviving samples take the full
// trilinear interpolation (8 taps, blocks resolved through the dense block
// index, cached across samples).
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/vsg.h"
#include "vsg_device.cuh"
#include "vsg_internal.h"
#include "vsg_raycast_core.cuh"

namespace vsg {

// One thread per pixel; a CTA covers 16x8 pixels as four 8x4 warp tiles.
__global__ void __launch_bounds__(128, 6) k_render(RenderArgs a) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    const int y = blockIdx.y * 8 + (warp >> 1) * 4 + (lane >> 3);
    if (x >= a.W || y >= a.H) return;
    render_pixel(a, x, y);
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
__global__ void __launch_bounds__(256) k_tile_bounds(RenderArgs a) {
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
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            atomicMax(glob, 0xFFFFFFFFu);  // nearest 0
            atomicMax(glob + 1, 0x7F800000u);  // farthest +inf
        }
        return;
    }
    const float zc = 0.5f * a.minD;
    const float mpx = 2.0f + 10.0f * e * (fabsf(a.fx) + fabsf(a.fy) + (float)a.W + (float)a.H);
    const float v = s.voxel;
    const uint32_t hw = s.ctr->high_water;
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < hw; b += gridDim.x * blockDim.x) {
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

// Exhaustive check of div_fixed against IEEE division for this voxel size:
// every float x with kDivTiny <= |x| < kDivRange, both signs.  One thread
// per bit pattern of |x|.
__global__ void k_verify_div(float v, float y, unsigned int* mismatches) {
    const uint32_t first = __float_as_uint(kDivTiny), limit = __float_as_uint(kDivRange);
    for (uint32_t u = first + blockIdx.x * blockDim.x + threadIdx.x; u < limit; u += gridDim.x * blockDim.x) {
        const float x = __uint_as_float(u);
        const float a = x / v, b = div_fixed(x, v, y);
        const float c = (-x) / v, d = div_fixed(-x, v, y);
        if (__float_as_uint(a) != __float_as_uint(b) || __float_as_uint(c) != __float_as_uint(d))
            atomicAdd(mismatches, 1u);
    }
}

int verify_fixed_division(float v, bool* ok) {
    *ok = false;
    unsigned int* d = nullptr;
    if (cudaMalloc(&d, sizeof(unsigned int)) != cudaSuccess) return VSG_ERR_OUT_OF_MEMORY;
    cudaMemset(d, 0, sizeof(unsigned int));
    const float y = 1.0f / v;
    int sms = 148;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_verify_div<<<sms * 8, 256>>>(v, y, d);
    unsigned int h = 1u;
    const cudaError_t e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return VSG_ERR_CUDA;
    *ok = h == 0u;
    return VSG_OK;
}

__global__ void k_count_touched(const uint8_t* touched, const SceneCounters* ctr, FrameCounters* f) {
    const uint32_t hw = ctr->high_water;
    uint32_t c = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < hw; i += gridDim.x * blockDim.x) c += touched[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(&f->blocks_read, c);
}

__global__ void k_render_begin(FrameCounters* f) { render_begin(f); }

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
    a.rec = r->record ? r->bracket : nullptr;
    a.touched = sc->timing.enabled ? sc->dev.block_touched : nullptr;
    a.t1x = (r->w + 7) / 8;
    a.t2x = (r->w + 63) / 64;
    a.n1 = a.t1x * ((r->h + 3) / 4);
    a.n2 = a.t2x * ((r->h + 31) / 32);
    a.bounds = r->bounds;
    if (a.touched) cudaMemsetAsync(a.touched, 0, (size_t)sc->dev.num_blocks, st);
    k_render_begin<<<1, 1, 0, st>>>(sc->dev.frame);
    dim3 grid((r->w + 15) / 16, (r->h + 7) / 8);
    timing_begin(sc, kSlotRender, st);
    cudaMemsetAsync(r->bounds, 0, sizeof(uint2) * (size_t)(a.n1 + a.n2 + 1), st);
    k_tile_bounds<<<sc->sm_count * 4, 256, 0, st>>>(a);
    k_render<<<grid, 128, 0, st>>>(a);
    timing_end(sc, kSlotRender, st);
    if (a.touched) k_count_touched<<<sc->sm_count * 2, 256, 0, st>>>(a.touched, sc->dev.ctr, sc->dev.frame);
    return cudaGetLastError() == cudaSuccess ? VSG_OK : VSG_ERR_CUDA;
}

}  // namespace vsg
