// vsg_points.cu -- voxel-wise surface-point extraction.
//
// Restates kernelExtractSurfacePoints / extractSurfacePointsCUDA /
// RayCastRender::extractSurfacePoints (RayCastRender.cu:683-910,
// RayCastRender.cpp:307-360): every voxel of an allocated block whose weight
// is non-zero and >= minWeight and whose SDF lies in [minSDF, maxSDF] yields
// one point -- the mean of the linear zero crossings towards its six
// neighbours (neighbours inside the block by index, outside through
// getVoxel at the centre +- one voxel, RayCastRender.cu:55-121), or its
// centre when there is none and |sdf| < 0.001 -- with its colour / 255 and
// the normalised central-difference SDF gradient at the point
// (computeNormalFromSDF, :629-677).  Arithmetic follows the reference
// operation by operation.
//
// Work layout: one CTA of 512 threads per pool block at a time (persistent
// grid); the block's voxels are staged in shared memory for the in-block
// neighbours, cross-block neighbours and the normal's six taps go through
// the dense block index; per block one CTA-wide scan and ONE atomic reserve
// the output range.  Blocks without a weighted voxel are skipped on their
// weight mask (every voxel would fail the weight test).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <new>
#include <vector>

#include "../../include/vsg.h"
#include "vsg_device.cuh"
#include "vsg_internal.h"

namespace vsg {
namespace {

constexpr int kPtThreads = 512;
constexpr int kPtWarps = kPtThreads / 32;

struct PtCounters {
    unsigned long long total;
    int total_i32;  // min(total, INT_MAX): the reference's int counter
    int pad;
};

// getVoxel (RayCastRender.cu:55-121): the voxel at the rounded position, or
// an empty one (sdf 0, weight 0) where no block is allocated.
__device__ __forceinline__ Voxel voxel_at(const SceneDev& s, float px, float py, float pz) {
    const float v = s.voxel;
    const float p[3] = {px / v, py / v, pz / v};
    int q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float sg = (p[a] > 0) ? 1.0f : ((p[a] < 0) ? -1.0f : 0.0f);
        q[a] = __float2int_rz(floorf(p[a] + 0.5f * sg));
    }
    const int ptr = block_ptr(s, q[0] >> 3, q[1] >> 3, q[2] >> 3);
    if (ptr < 0) return Voxel{0.0f, 0u};
    return s.voxels[(size_t)ptr * kVoxPerBlock + (q[0] & 7) + (q[1] & 7) * kBlock + (q[2] & 7) * kBlock * kBlock];
}

__global__ void __launch_bounds__(kPtThreads) k_extract_points(SceneDev s, float min_sdf, float max_sdf,
                                                               uint32_t min_w, float4* __restrict__ pos,
                                                               float4* __restrict__ col, float4* __restrict__ nrm,
                                                               PtCounters* ctr, int max_pts) {
    __shared__ Voxel vx[kVoxPerBlock];
    __shared__ int warp_tot[kPtWarps];
    __shared__ unsigned long long s_base;
    const uint32_t hw = s.ctr->high_water;
    const int t = threadIdx.x;
    const int lx = t & 7, ly = (t >> 3) & 7, lz = t >> 6;
    const int lane = t & 31, warp = t >> 5;
    const float v = s.voxel;
    for (uint32_t b = blockIdx.x; b < hw; b += gridDim.x) {
        const unsigned long long key = s.block_key[b];
        if (key == kKeyEmpty || key == kKeyTomb) continue;
        if (s.block_fresh[b] || s.block_wmask[b] == 0ull) continue;
        __syncthreads();  // previous block's readers of vx done
        vx[t] = s.voxels[(size_t)b * kVoxPerBlock + t];
        __syncthreads();
        int bx, by, bz;
        unpack_key(key, bx, by, bz);
        const Voxel me = vx[t];
        const uint32_t w = me.rgbw >> 24;
        bool out = false;
        float iso[3] = {0.0f, 0.0f, 0.0f};
        if (w != 0u && w >= min_w && !(me.sdf < min_sdf || me.sdf > max_sdf)) {
            // voxel centre, RayCastRender.cu:713-717, 740-744
            const float c[3] = {(float)(bx * kBlock) * v + ((float)lx + 0.5f) * v,
                                (float)(by * kBlock) * v + ((float)ly + 0.5f) * v,
                                (float)(bz * kBlock) * v + ((float)lz + 0.5f) * v};
            const int l[3] = {lx, ly, lz};
            float acc[3] = {0.0f, 0.0f, 0.0f};
            int nv = 0;
#pragma unroll
            for (int d = 0; d < 6; ++d) {
                const int axis = d >> 1;
                const int sgn = (d & 1) ? -1 : 1;  // x+, x-, y+, y-, z+, z-
                const int nl = l[axis] + sgn;
                Voxel nb;
                if (nl < 0 || nl >= kBlock) {
                    float q[3] = {c[0], c[1], c[2]};
                    q[axis] = c[axis] + (float)sgn * v;
                    nb = voxel_at(s, q[0], q[1], q[2]);
                } else {
                    int ll[3] = {lx, ly, lz};
                    ll[axis] = nl;
                    nb = vx[ll[0] + ll[1] * kBlock + ll[2] * kBlock * kBlock];
                }
                if ((nb.rgbw >> 24) == 0u) continue;
                if ((me.sdf < 0.0f && nb.sdf > 0.0f) || (me.sdf > 0.0f && nb.sdf < 0.0f)) {
                    const float tt = me.sdf / (me.sdf - nb.sdf);
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const float dir = a == axis ? (float)sgn : 0.0f;
                        acc[a] += c[a] + dir * v * tt;
                    }
                    ++nv;
                }
            }
            if (nv == 0) {
                if (fabsf(me.sdf) < 0.001f) {
                    iso[0] = c[0];
                    iso[1] = c[1];
                    iso[2] = c[2];
                    out = true;
                }
            } else {
#pragma unroll
                for (int a = 0; a < 3; ++a) iso[a] = acc[a] / (float)nv;
                out = true;
            }
        }
        // CTA-wide exclusive scan of the per-voxel point flags
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, out);
        if (lane == 0) warp_tot[warp] = __popc(bal);
        __syncthreads();
        int before = 0, total = 0;
#pragma unroll
        for (int k = 0; k < kPtWarps; ++k) {
            const int c = warp_tot[k];
            before += k < warp ? c : 0;
            total += c;
        }
        if (t == 0) {
            unsigned long long base = 0ull;
            if (total) {
                base = atomicAdd(&ctr->total, (unsigned long long)total);
                const unsigned long long end = base + (unsigned long long)total;
                atomicMax(&ctr->total_i32, end > 0x7FFFFFFFull ? 0x7FFFFFFF : (int)end);
            }
            s_base = base;
        }
        __syncthreads();
        if (!out) continue;
        const unsigned long long o = s_base + (unsigned long long)(before + __popc(bal & ((1u << lane) - 1u)));
        if (o >= (unsigned long long)max_pts) continue;
        // computeNormalFromSDF, RayCastRender.cu:629-677
        const float eps = v * 0.5f;
        float g[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float q1[3] = {iso[0], iso[1], iso[2]}, q0[3] = {iso[0], iso[1], iso[2]};
            q1[a] = iso[a] + eps;
            q0[a] = iso[a] - eps;
            const Voxel v1 = voxel_at(s, q1[0], q1[1], q1[2]);
            const Voxel v0 = voxel_at(s, q0[0], q0[1], q0[2]);
            g[a] = ((v1.rgbw >> 24) > 0u && (v0.rgbw >> 24) > 0u) ? (v1.sdf - v0.sdf) / (2.0f * eps) : 0.0f;
        }
        const float len = sqrtf(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
        if (len > 1e-6f) {
            g[0] /= len;
            g[1] /= len;
            g[2] /= len;
        }
        pos[o] = make_float4(iso[0], iso[1], iso[2], 1.0f);
        col[o] = make_float4((float)(me.rgbw & 0xFFu) / 255.0f, (float)((me.rgbw >> 8) & 0xFFu) / 255.0f,
                             (float)((me.rgbw >> 16) & 0xFFu) / 255.0f, 1.0f);
        nrm[o] = make_float4(g[0], g[1], g[2], 0.0f);
    }
}

}  // namespace

struct Points {
    float4* pos = nullptr;
    float4* col = nullptr;
    float4* nrm = nullptr;
    PtCounters* ctr = nullptr;
    int max_pts = 0;
    int device = 0;
};

}  // namespace vsg

struct vsg_points {
    vsg::Points impl;
};

namespace {

void free_points(vsg::Points& p) {
    cudaFree(p.pos);
    cudaFree(p.col);
    cudaFree(p.nrm);
    cudaFree(p.ctr);
}

}  // namespace

extern "C" {

int vsg_points_create(int max_points, vsg_points** out) {
    if (!out || max_points <= 0) return VSG_ERR_INVALID_ARG;
    *out = nullptr;
    vsg_points* m = new (std::nothrow) vsg_points();
    if (!m) return VSG_ERR_OUT_OF_MEMORY;
    vsg::Points& p = m->impl;
    cudaGetDevice(&p.device);
    const size_t bytes = (size_t)max_points * sizeof(float4);
    if (cudaMalloc(&p.pos, bytes) != cudaSuccess || cudaMalloc(&p.col, bytes) != cudaSuccess ||
        cudaMalloc(&p.nrm, bytes) != cudaSuccess || cudaMalloc(&p.ctr, sizeof(vsg::PtCounters)) != cudaSuccess ||
        cudaMemset(p.ctr, 0, sizeof(vsg::PtCounters)) != cudaSuccess) {
        free_points(p);
        delete m;
        return VSG_ERR_OUT_OF_MEMORY;
    }
    p.max_pts = max_points;
    *out = m;
    return VSG_OK;
}

int vsg_points_destroy(vsg_points* m) {
    if (!m) return VSG_ERR_INVALID_ARG;
    free_points(m->impl);
    delete m;
    return VSG_OK;
}

int vsg_extract_points(vsg_scene* s, vsg_points* m, float min_sdf, float max_sdf, uint32_t min_weight,
                       vsg_stream_t stream) {
    if (!s || !m) return VSG_ERR_INVALID_ARG;
    vsg::Scene* sc = &s->impl;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != sc->device || dev != m->impl.device) return VSG_ERR_INVALID_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(m->impl.ctr, 0, sizeof(vsg::PtCounters), st) != cudaSuccess) return VSG_ERR_CUDA;
    vsg::timing_begin(sc, vsg::kSlotExtractPoints, st);
    vsg::k_extract_points<<<sc->sm_count * 3, vsg::kPtThreads, 0, st>>>(sc->dev, min_sdf, max_sdf, min_weight,
                                                                        m->impl.pos, m->impl.col, m->impl.nrm,
                                                                        m->impl.ctr, m->impl.max_pts);
    vsg::timing_end(sc, vsg::kSlotExtractPoints, st);
    return cudaGetLastError() == cudaSuccess ? VSG_OK : VSG_ERR_CUDA;
}

int vsg_points_count(const vsg_points* m, int64_t* count) {
    if (!m || !count) return VSG_ERR_INVALID_ARG;
    int dev = -1;  // the synchronisation below waits for the current device only
    if (cudaGetDevice(&dev) != cudaSuccess || dev != m->impl.device) return VSG_ERR_INVALID_ARG;
    if (cudaDeviceSynchronize() != cudaSuccess) return VSG_ERR_CUDA;
    vsg::PtCounters c{};
    if (cudaMemcpy(&c, m->impl.ctr, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess) return VSG_ERR_CUDA;
    *count = (int64_t)c.total;
    return VSG_OK;
}

int vsg_points_buffers(const vsg_points* m, float** positions, float** colors, float** normals, int** count_dev,
                       int* max_points) {
    if (!m) return VSG_ERR_INVALID_ARG;
    if (positions) *positions = reinterpret_cast<float*>(m->impl.pos);
    if (colors) *colors = reinterpret_cast<float*>(m->impl.col);
    if (normals) *normals = reinterpret_cast<float*>(m->impl.nrm);
    if (count_dev) *count_dev = &m->impl.ctr->total_i32;
    if (max_points) *max_points = m->impl.max_pts;
    return VSG_OK;
}

int vsg_points_download(const vsg_points* m, float* positions, float* colors, float* normals, int64_t* count) {
    if (!m) return VSG_ERR_INVALID_ARG;
    int64_t n = 0;
    const int rc = vsg_points_count(m, &n);
    if (rc != VSG_OK) return rc;
    if (count) *count = n;
    const size_t bytes = (size_t)(n < m->impl.max_pts ? n : m->impl.max_pts) * sizeof(float4);
    if (bytes && positions && cudaMemcpy(positions, m->impl.pos, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        return VSG_ERR_CUDA;
    if (bytes && colors && cudaMemcpy(colors, m->impl.col, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        return VSG_ERR_CUDA;
    if (bytes && normals && cudaMemcpy(normals, m->impl.nrm, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        return VSG_ERR_CUDA;
    return VSG_OK;
}

// saveExtractedSurfacePointsPLY (RayCastRender.cpp:370-446): ASCII PLY of the
// written points with finite positions; colour channels clamped to [0, 1]
// and rounded to 0..255 (non-finite -> 255).
int vsg_points_save_ply(const vsg_points* m, const char* path) {
    return vsg::host_guard([&]() -> int {
        if (!m || !path) return VSG_ERR_INVALID_ARG;
        int64_t n = 0;
        int rc = vsg_points_count(m, &n);
        if (rc != VSG_OK) return rc;
        const size_t k = (size_t)(n < m->impl.max_pts ? n : m->impl.max_pts);
        std::vector<float4> P(k), C(k), N(k);
        rc = vsg_points_download(m, reinterpret_cast<float*>(P.data()), reinterpret_cast<float*>(C.data()),
                                 reinterpret_cast<float*>(N.data()), nullptr);
        if (rc != VSG_OK) return rc;
        size_t valid = 0;
        for (size_t i = 0; i < k; ++i)
            if (std::isfinite(P[i].x) && std::isfinite(P[i].y) && std::isfinite(P[i].z)) ++valid;
        FILE* f = std::fopen(path, "w");
        if (!f) return VSG_ERR_INVALID_ARG;
        std::fprintf(f,
                     "ply\nformat ascii 1.0\ncomment Generated by RayCastRender::extractSurfacePoints\n"
                     "element vertex %zu\nproperty float x\nproperty float y\nproperty float z\n"
                     "property float nx\nproperty float ny\nproperty float nz\n"
                     "property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n",
                     valid);
        auto channel = [](float c) -> int {
            if (!std::isfinite(c)) return 255;
            c = c < 0.0f ? 0.0f : (c > 1.0f ? 1.0f : c);
            return static_cast<int>(c * 255.0f + 0.5f);
        };
        for (size_t i = 0; i < k; ++i) {
            if (!(std::isfinite(P[i].x) && std::isfinite(P[i].y) && std::isfinite(P[i].z))) continue;
            std::fprintf(f, "%g %g %g %g %g %g %d %d %d\n", P[i].x, P[i].y, P[i].z, N[i].x, N[i].y, N[i].z,
                         channel(C[i].x), channel(C[i].y), channel(C[i].z));
        }
        return std::fclose(f) == 0 ? VSG_OK : VSG_ERR_INVALID_ARG;
    });
}

}  // extern "C"
