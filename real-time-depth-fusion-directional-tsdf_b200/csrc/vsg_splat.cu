// vsg_splat.cu -- point cloud -> depth / point / normal / colour maps
// (CustomDepthMapGenerator::generateFromPointCloud, CustomDepthMapGenerator.
// cpp:81-222, the producer of the point maps the fusion path consumes).
//
// The reference projects each point with z > 0 (perspective, :550-556),
// keeps it when the projection lies in [0, w) x [0, h), and writes pixel
// (floor u, floor v) in input order, so the last point wins the pixel; a
// point's normal and colour are written only when the point has one
// (i < normals.size(), i < colors.size()).  Without normals the depth map's
// fallback normals follow (:163-209).  Its CUDA counterpart
// (CUDADepthMapData.cu:9-53) keeps the nearest point with an unguarded
// read-compare-write that races.
//
// Here, race-free and deterministic on the GPU:
//   k_splat    one thread per point: 64-bit atomicMax of (index + 1) per
//              pixel (last-wins), or atomicMin of (z bits << 32 | ~index)
//              (nearest point, later index on equal z); in last-wins mode
//              two more 32-bit maxima pick the last point with a normal and
//              the last with a colour
//   k_resolve  one thread per pixel: writes the winners' attributes
//   k_normals  (no normals given) the generator's fallback on the depth map
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/vsg.h"
#include "vsg_normals.cuh"

namespace {

struct SplatWork {
    unsigned long long* key;  // per pixel
    uint32_t* nwin;           // last point with a normal (+1), last-wins mode
    uint32_t* cwin;           // last point with a colour (+1), last-wins mode
    float* depth;             // resolved depth (for the normal fallback)
};

__global__ void __launch_bounds__(256) k_splat(const float* __restrict__ pts, long long n, long long n_nrm,
                                               long long n_col, int W, int H, float fx, float fy, float cx, float cy,
                                               float zmin, float zmax, int mode, SplatWork wk) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float x = pts[3 * i], y = pts[3 * i + 1], z = pts[3 * i + 2];
        if (z <= 0.0f) continue;                 // :114
        if (z < zmin || z > zmax) continue;      // optional depth range
        const float u = (x * fx / z) + cx;       // :553-556
        const float v = (y * fy / z) + cy;
        if (!(u >= 0.0f && u < (float)W && v >= 0.0f && v < (float)H)) continue;  // :586-587
        const int px = (int)floorf(u), py = (int)floorf(v);
        if (px < 0 || py < 0 || px >= W || py >= H) continue;  // :142
        const size_t p = (size_t)py * W + px;
        if (mode == VSG_SPLAT_NEAREST) {
            const unsigned long long k =
                ((unsigned long long)__float_as_uint(z) << 32) | (unsigned long long)(0xFFFFFFFFu - (uint32_t)i);
            atomicMin(wk.key + p, k);
        } else {
            atomicMax(wk.key + p, (unsigned long long)(i + 1));
            if (i < n_nrm) atomicMax(wk.nwin + p, (uint32_t)(i + 1));
            if (i < n_col) atomicMax(wk.cwin + p, (uint32_t)(i + 1));
        }
    }
}

__global__ void __launch_bounds__(256) k_resolve(const float* __restrict__ pts, const float* __restrict__ nrm,
                                                 long long n_nrm, const uint8_t* __restrict__ col, long long n_col,
                                                 int npx, int mode, SplatWork wk, float* depth, float* pm, float* nm,
                                                 uint8_t* cm, unsigned int* n_valid) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    bool hit = false;
    if (p < npx) {
        const unsigned long long k = wk.key[p];
        long long j = -1, jn = -1, jc = -1;
        if (mode == VSG_SPLAT_NEAREST) {
            if (k != ~0ull) {
                j = (long long)(0xFFFFFFFFu - (uint32_t)(k & 0xFFFFFFFFull));
                jn = j < n_nrm ? j : -1;
                jc = j < n_col ? j : -1;
            }
        } else if (k != 0ull) {
            j = (long long)k - 1;
            jn = (long long)wk.nwin[p] - 1;
            jc = (long long)wk.cwin[p] - 1;
        }
        hit = j >= 0;
        const float px = hit ? pts[3 * j] : 0.0f, py = hit ? pts[3 * j + 1] : 0.0f, pz = hit ? pts[3 * j + 2] : 0.0f;
        wk.depth[p] = pz;
        if (depth) depth[p] = pz;
        if (pm) {
            pm[3 * p] = px;
            pm[3 * p + 1] = py;
            pm[3 * p + 2] = pz;
        }
        if (nm && n_nrm > 0) {
            nm[3 * p] = jn >= 0 ? nrm[3 * jn] : 0.0f;
            nm[3 * p + 1] = jn >= 0 ? nrm[3 * jn + 1] : 0.0f;
            nm[3 * p + 2] = jn >= 0 ? nrm[3 * jn + 2] : 0.0f;
        }
        if (cm) {
            cm[3 * p] = jc >= 0 ? col[3 * jc] : 0;
            cm[3 * p + 1] = jc >= 0 ? col[3 * jc + 1] : 0;
            cm[3 * p + 2] = jc >= 0 ? col[3 * jc + 2] : 0;
        }
    }
    if (n_valid) {
        const unsigned m = __ballot_sync(0xFFFFFFFFu, hit);
        if ((threadIdx.x & 31) == 0 && m) atomicAdd(n_valid, (unsigned)__popc(m));
    }
}

__global__ void k_normals(const float* __restrict__ depth, int W, int H, float fx, float fy, float cx, float cy,
                          float* __restrict__ nm) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t i = (size_t)y * W + x;
    const float3 n = vsg::depth_normal(depth, W, H, x, y, fx, fy, cx, cy);
    nm[3 * i] = n.x;
    nm[3 * i + 1] = n.y;
    nm[3 * i + 2] = n.z;
}

}  // namespace

extern "C" {

int vsg_splat_points(const float* points, int64_t n_points, const float* normals, int64_t n_normals,
                     const uint8_t* colors, int64_t n_colors, int w, int h, float fx, float fy, float cx, float cy,
                     float min_depth, float max_depth, int mode, float* depth, float* pointmap, float* normalmap,
                     uint8_t* colormap, int64_t* n_valid, vsg_stream_t stream) {
    if (w <= 0 || h <= 0 || (long long)w * h > (1ll << 30) || n_points < 0 || n_normals < 0 || n_colors < 0)
        return VSG_ERR_INVALID_ARG;
    if (mode != VSG_SPLAT_LAST && mode != VSG_SPLAT_NEAREST) return VSG_ERR_INVALID_ARG;
    if ((n_points && !points) || (n_normals && !normals) || (n_colors && !colors)) return VSG_ERR_INVALID_ARG;
    if (n_points >= 0xFFFFFFFFll) return VSG_ERR_TOO_LARGE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t npx = (size_t)w * h;
    unsigned char* buf = nullptr;
    const size_t bytes = npx * (8 + 4 + 4 + 4) + 16;
    if (cudaMallocAsync(reinterpret_cast<void**>(&buf), bytes, st) != cudaSuccess) return VSG_ERR_OUT_OF_MEMORY;
    SplatWork wk;
    wk.key = reinterpret_cast<unsigned long long*>(buf);
    wk.nwin = reinterpret_cast<uint32_t*>(buf + npx * 8);
    wk.cwin = wk.nwin + npx;
    wk.depth = reinterpret_cast<float*>(wk.cwin + npx);
    unsigned int* cnt = reinterpret_cast<unsigned int*>(wk.depth + npx);
    int rc = VSG_OK;
    if (cudaMemsetAsync(wk.key, mode == VSG_SPLAT_NEAREST ? 0xFF : 0x00, npx * 8, st) != cudaSuccess ||
        cudaMemsetAsync(wk.nwin, 0, npx * 8, st) != cudaSuccess || cudaMemsetAsync(cnt, 0, 4, st) != cudaSuccess)
        rc = VSG_ERR_CUDA;
    if (rc == VSG_OK) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const long long want = (n_points + 255) / 256;
        const int grid = (int)(want < (long long)sms * 16 ? (want > 0 ? want : 1) : (long long)sms * 16);
        if (n_points > 0)
            k_splat<<<grid, 256, 0, st>>>(points, n_points, n_normals, n_colors, w, h, fx, fy, cx, cy, min_depth,
                                          max_depth, mode, wk);
        k_resolve<<<(unsigned)((npx + 255) / 256), 256, 0, st>>>(points, normals, n_normals, colors, n_colors,
                                                                 (int)npx, mode, wk, depth, pointmap, normalmap,
                                                                 colormap, n_valid ? cnt : nullptr);
        if (normalmap && n_normals == 0)
            k_normals<<<dim3((w + 31) / 32, (h + 7) / 8), dim3(32, 8), 0, st>>>(wk.depth, w, h, fx, fy, cx, cy,
                                                                             normalmap);
        if (cudaGetLastError() != cudaSuccess) rc = VSG_ERR_CUDA;
    }
    if (rc == VSG_OK && n_valid) {
        unsigned int v = 0;
        if (cudaMemcpyAsync(&v, cnt, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            rc = VSG_ERR_CUDA;
        *n_valid = v;
    }
    cudaFreeAsync(buf, st);
    return rc;
}

}  // extern "C"
