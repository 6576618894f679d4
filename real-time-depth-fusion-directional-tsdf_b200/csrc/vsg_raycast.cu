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
// index, cached across samples).  Before the march, k_tile_bounds records per
// pixel tile the nearest and farthest distance at which any weighted block
// can be read; each ray starts at the first and stops after the second
// (tile_bounds_range, apply_bounds).
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/vsg.h"
#include "vsg_device.cuh"
#include "vsg_internal.h"
#include "vsg_raycast_core.cuh"

namespace vsg {

// One thread per pixel; a CTA covers 16x8 pixels as four 8x4 warp tiles, the
// CTAs taking the tiles in the order k_tile_order wrote (longest march range
// first).  kCountSkips: the scene's march statistics are on (render_pixel).
// Seven resident CTAs per SM (72 registers, no spills) for the production
// caster: 0.795 / 1.467 ms per tabletop / room frame against 0.799 / 1.552
// at six; the counting caster needs 80 registers.
template <bool kCountSkips>
__global__ void __launch_bounds__(128, kCountSkips ? 6 : 7) k_render(RenderArgs a, const uint32_t* __restrict__ order, int gx) {
    const uint32_t t = __ldg(order + blockIdx.x);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = (int)(t % (uint32_t)gx) * 16 + (warp & 1) * 8 + (lane & 7);
    const int y = (int)(t / (uint32_t)gx) * 8 + (warp >> 1) * 4 + (lane >> 3);
    if (x >= a.W || y >= a.H) return;
    render_pixel<kCountSkips>(a, x, y);
}

// Ray-cast tile order, longest march first (tile_bucket); one CTA: bucket
// counts in shared memory, then a scatter.
__global__ void __launch_bounds__(1024) k_tile_order(RenderArgs a, uint32_t* order, int gx, int n) {
    __shared__ unsigned hist[kOrderBuckets], next[kOrderBuckets];
    if (threadIdx.x < kOrderBuckets) hist[threadIdx.x] = 0u;
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) atomicAdd(&hist[tile_bucket(a, t % gx, t / gx)], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned s = 0;
        for (int b = kOrderBuckets - 1; b >= 0; --b) {  // heaviest bucket first
            next[b] = s;
            s += hist[b];
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) order[atomicAdd(&next[tile_bucket(a, t % gx, t / gx)], 1u)] = (uint32_t)t;
}

// The ray-distance bounds of one render (tile_bounds_range), one thread per
// pool block.
__global__ void __launch_bounds__(256) k_tile_bounds(RenderArgs a) {
    tile_bounds_range(a, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
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
    a.step = r->step;
    a.depth = r->depth;
    a.pos = r->position;
    a.col = r->color;
    a.nrm = r->normal;
    a.rec = r->record ? r->bracket : nullptr;
    a.touched = sc->march_stats ? sc->dev.block_touched : nullptr;
    a.t1x = (r->w + 7) / 8;
    a.t2x = (r->w + 63) / 64;
    a.n1 = a.t1x * ((r->h + 3) / 4);
    a.n2 = a.t2x * ((r->h + 31) / 32);
    a.bounds = r->bounds;
    if (a.touched) cudaMemsetAsync(a.touched, 0, (size_t)sc->dev.num_blocks, st);
    k_render_begin<<<1, 1, 0, st>>>(sc->dev.frame);
    const int gx = (r->w + 15) / 16, ntiles = gx * ((r->h + 7) / 8);
    timing_begin(sc, kSlotRender, st);
    cudaMemsetAsync(r->bounds, 0, sizeof(uint2) * (size_t)(a.n1 + a.n2 + 1), st);
    k_tile_bounds<<<sc->sm_count * 4, 256, 0, st>>>(a);
    k_tile_order<<<1, 1024, 0, st>>>(a, r->tile_order, gx, ntiles);
    if (sc->march_stats)
        k_render<true><<<ntiles, 128, 0, st>>>(a, r->tile_order, gx);
    else
        k_render<false><<<ntiles, 128, 0, st>>>(a, r->tile_order, gx);
    timing_end(sc, kSlotRender, st);
    if (a.touched) k_count_touched<<<sc->sm_count * 2, 256, 0, st>>>(a.touched, sc->dev.ctr, sc->dev.frame);
    return cudaGetLastError() == cudaSuccess ? VSG_OK : VSG_ERR_CUDA;
}

}  // namespace vsg
