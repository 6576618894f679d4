// vsg_integ_adjoint.cu -- gradient of one frame's TSDF integration with
// respect to the frame's camera pose and point map (no counterpart in the
// reference).
//
// integrateDepthMapIntoBlocksKernel (VoxelScene.cu:954-1126) updates a voxel
// at world centre w from the pixel its centre projects to:
//   P = T p (the pixel's camera-space point p, world), s = +-|w - P| (minus
//   when w is nearer the camera than P), kept when |s| <= truncation;
//   sdf' = (sdf W + s) / (W + 1),  W' = min(255, W + 1).
// With the discrete decisions fixed (the pixel, the sign, the truncation
// test), sdf' is smooth in T and p:
//   d sdf' / d sdf = W / (W + 1),  d sdf' / d P = -sign (w - P) / |w - P| / (W + 1),
//   P = R p + t.
// vsg_integrate_backward runs right after the vsg_integrate of that frame:
// it revisits every allocated block, retraces each voxel's projection and
// tests with the forward's FP32 operations, and for the voxels the frame
// updated turns dL/dsdf' (the caller's buffer, indexed like the pool) into
// dL/dsdf before the frame (in place), dL/dT (deterministic double
// reduction) and dL/dp (float atomics per pixel).  The weight before the
// frame is the stored weight minus one; a voxel found at the cap (255) is
// taken to have reached it with this frame.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "../../include/vsg.h"
#include "vsg_device.cuh"
#include "vsg_internal.h"

namespace vsg {
namespace {

constexpr int kIbWarps = 8;  // warps per CTA

struct IntegBackArgs {
    SceneDev s;
    const float* pm;
    int W, H;
    float trunc;
    Pose pose;
    float fx, fy, cx, cy;
    float* g_sdf;
    float* g_pm;
    double* partials;  // per warp 12
    unsigned int* n_upd;
};

__global__ void __launch_bounds__(kIbWarps * 32) k_integrate_backward(IntegBackArgs a) {
    const SceneDev& s = a.s;
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * kIbWarps + (threadIdx.x >> 5);
    const int nw = gridDim.x * kIbWarps;
    const uint32_t hw = s.ctr->high_water;
    const float* T = a.pose.T;
    const float v = s.voxel;
    const float camx = T[3], camy = T[7], camz = T[11];
    const float t = a.trunc;
    double gT[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) gT[i] = 0.0;
    unsigned int n_upd = 0;
    for (uint32_t b = gw; b < hw; b += nw) {
        const unsigned long long key = s.block_key[b];
        if (key == kKeyEmpty || key == kKeyTomb) continue;
        int bx, by, bz;
        unpack_key(key, bx, by, bz);
        // the block's stored parent pixel, as the forward chose it
        // (VoxelScene.cu:1015-1035)
        int ppix = -1;
        if (const unsigned long long pt = s.block_parent[b]) {
            const int px = (int)(pt & 0xFFFFu), py = (int)((pt >> 16) & 0xFFFFu);
            if (px < a.W && py < a.H) {
                const size_t q = (size_t)py * a.W + px;
                if (a.pm[3 * q] != 0.0f || a.pm[3 * q + 1] != 0.0f || a.pm[3 * q + 2] != 0.0f) ppix = (int)q;
            }
        }
        const int lx = lane & 7;
        const float wx = (float)(int)((unsigned)bx * 8u + (unsigned)lx) * v;
        const float rx = wx - T[3];
        for (int k = 0; k < 16; ++k) {
            // the forward's projection and tests, VoxelScene.cu:984-1066
            const int ly = (lane >> 3) + ((k & 1) << 2);
            const int lz = k >> 1;
            const float wy = (float)(int)((unsigned)by * 8u + (unsigned)ly) * v;
            const float wz = (float)(int)((unsigned)bz * 8u + (unsigned)lz) * v;
            const float ry = wy - T[7], rz = wz - T[11];
            const float cxp = T[0] * rx + T[4] * ry + T[8] * rz;
            const float cyp = T[1] * rx + T[5] * ry + T[9] * rz;
            const float czp = T[2] * rx + T[6] * ry + T[10] * rz;
            const float sx = cxp * a.fx / czp + a.cx;
            const float sy = cyp * a.fy / czp + a.cy;
            const int ix = __float2int_rz(sx + 0.5f), iy = __float2int_rz(sy + 0.5f);
            if (ppix < 0 && !(ix >= 0 && ix < a.W && iy >= 0 && iy < a.H)) continue;
            const size_t pix = ppix >= 0 ? (size_t)ppix : (size_t)iy * a.W + ix;
            const float p0 = a.pm[3 * pix], p1 = a.pm[3 * pix + 1], p2 = a.pm[3 * pix + 2];
            if (p0 == 0.0f && p1 == 0.0f && p2 == 0.0f) continue;
            // depthPos_world and cameraDist, as the allocation kernel forms them
            const float Px = T[0] * p0 + T[1] * p1 + T[2] * p2 + T[3];
            const float Py = T[4] * p0 + T[5] * p1 + T[6] * p2 + T[7];
            const float Pz = T[8] * p0 + T[9] * p1 + T[10] * p2 + T[11];
            const float ex = Px - T[3], ey = Py - T[7], ez = Pz - T[11];
            const float pdist = sqrtf(ex * ex + ey * ey + ez * ez);
            const float dx = wx - Px, dy = wy - Py, dz = wz - Pz;
            float sdf = sqrtf(dx * dx + dy * dy + dz * dz);
            const float vdist =
                sqrtf((wx - camx) * (wx - camx) + (wy - camy) * (wy - camy) + (wz - camz) * (wz - camz));
            const bool neg = vdist < pdist;
            if (neg) sdf = -sdf;
            if (sdf < -t || sdf > t) continue;
            // updated by the frame
            const size_t idx = (size_t)b * kVoxPerBlock + k * 32 + lane;
            const uint32_t wn = s.voxels[idx].rgbw >> 24;
            const double w_old = wn > 0u ? (double)(wn - 1u) : 0.0;
            const double g = a.g_sdf[idx];
            const double gs = g / (w_old + 1.0);      // dL / d(frame sdf)
            a.g_sdf[idx] = (float)(g * w_old / (w_old + 1.0));
            ++n_upd;
            const double Dx = (double)wx - ((double)T[0] * p0 + (double)T[1] * p1 + (double)T[2] * p2 + T[3]);
            const double Dy = (double)wy - ((double)T[4] * p0 + (double)T[5] * p1 + (double)T[6] * p2 + T[7]);
            const double Dz = (double)wz - ((double)T[8] * p0 + (double)T[9] * p1 + (double)T[10] * p2 + T[11]);
            const double len = sqrt(Dx * Dx + Dy * Dy + Dz * Dz);
            if (!(len > 0.0)) continue;
            // s = sign |w - P|: d s / d P = -sign (w - P) / |w - P|
            const double sg = neg ? -1.0 : 1.0;
            const double gP[3] = {-gs * sg * Dx / len, -gs * sg * Dy / len, -gs * sg * Dz / len};
            const double p[3] = {p0, p1, p2};
#pragma unroll
            for (int i = 0; i < 3; ++i) {
#pragma unroll
                for (int j = 0; j < 3; ++j) gT[4 * i + j] += gP[i] * p[j];
                gT[4 * i + 3] += gP[i];
            }
            if (a.g_pm) {
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const double gp = gP[0] * T[j] + gP[1] * T[4 + j] + gP[2] * T[8 + j];  // R^T gP
                    atomicAdd(a.g_pm + 3 * pix + j, (float)gp);
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        double x = gT[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, o);
        if (lane == 0) a.partials[(size_t)gw * 12 + i] = x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_upd += __shfl_xor_sync(0xFFFFFFFFu, n_upd, o);
    if (lane == 0 && n_upd) atomicAdd(a.n_upd, n_upd);
}

__global__ void k_reduce_partials(const double* partials, int n, double* out) {
    __shared__ double red[12][32];
    const int i = threadIdx.x / 32, lane = threadIdx.x % 32;  // 384 threads: 12 x 32
    double s = 0.0;
    for (int k = lane; k < n; k += 32) s += partials[(size_t)k * 12 + i];
    red[i][lane] = s;
    __syncthreads();
    if (lane == 0) {
        double t = 0.0;
        for (int k = 0; k < 32; ++k) t += red[i][k];
        out[i] = t;
    }
}

}  // namespace
}  // namespace vsg

extern "C" {

int vsg_integrate_backward(vsg_scene* s, const float* pointmap, int w, int h, float truncation, const float pose[16],
                           float fx, float fy, float cx, float cy, float* grad_sdf, double* grad_pose,
                           float* grad_pointmap, uint32_t* n_updated, vsg_stream_t stream) {
    if (!s || !pointmap || !pose || !grad_sdf || !grad_pose || w <= 0 || h <= 0) return VSG_ERR_INVALID_ARG;
    vsg::Scene* sc = &s->impl;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != sc->device) return VSG_ERR_INVALID_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int ctas = sc->sm_count * 4;
    const int warps = ctas * vsg::kIbWarps;
    double* partials = nullptr;
    unsigned int* cnt = nullptr;
    // a work buffer per call: warps x 12 doubles (~450 KB) and a counter
    if (cudaMallocAsync(&partials, (size_t)warps * 12 * sizeof(double) + 16, st) != cudaSuccess)
        return VSG_ERR_OUT_OF_MEMORY;
    cnt = reinterpret_cast<unsigned int*>(partials + (size_t)warps * 12);
    vsg::IntegBackArgs a;
    std::memset(&a, 0, sizeof(a));
    a.s = sc->dev;
    a.pm = pointmap;
    a.W = w;
    a.H = h;
    a.trunc = truncation;
    std::memcpy(a.pose.T, pose, sizeof(a.pose.T));
    a.fx = fx;
    a.fy = fy;
    a.cx = cx;
    a.cy = cy;
    a.g_sdf = grad_sdf;
    a.g_pm = grad_pointmap;
    a.partials = partials;
    a.n_upd = cnt;
    int rc = VSG_OK;
    if (cudaMemsetAsync(cnt, 0, sizeof(unsigned int), st) != cudaSuccess) rc = VSG_ERR_CUDA;
    if (rc == VSG_OK) {
        vsg::k_integrate_backward<<<ctas, vsg::kIbWarps * 32, 0, st>>>(a);
        vsg::k_reduce_partials<<<1, 384, 0, st>>>(partials, warps, grad_pose);
        if (cudaGetLastError() != cudaSuccess) rc = VSG_ERR_CUDA;
    }
    if (rc == VSG_OK && n_updated) {
        if (cudaMemcpyAsync(n_updated, cnt, sizeof(unsigned int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            rc = VSG_ERR_CUDA;
    }
    cudaFreeAsync(partials, st);
    return rc;
}

}  // extern "C"
