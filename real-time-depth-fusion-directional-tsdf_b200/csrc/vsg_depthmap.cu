// vsg_depthmap.cu -- depth image -> camera-space point map (and normals).
//
// The reference's fusion path consumes point maps produced upstream
// (CustomDepthMapGenerator::generateFromPointCloud, CustomDepthMapGenerator.
// cpp:81-222).  For callers with a depth image instead of a point cloud this
// back-projects every pixel, p = ((x - cx) d / fx, (y - cy) d / fy, d), the
// same expression the generator's normal computation uses (:170-193); pixels
// whose depth is not a positive finite number become (0,0,0), the invalid
// point.  Normals follow the generator's fallback (:163-209): for interior
// pixels with depth > 0, the normalised cross product of (right - centre)
// and (down - centre); every other pixel gets (0,0,0).
//
// One thread per pixel, 32x8 pixel tiles: the depth reads of a warp are one
// 128-byte row segment, the right and down neighbours come from L1.
#include <cuda_runtime.h>

#include "../../include/vsg.h"
#include "vsg_normals.cuh"

namespace {

using vsg::backproject;

__global__ void k_depth_to_maps(const float* __restrict__ depth, int W, int H, float fx, float fy, float cx,
                                float cy, float* __restrict__ pm, float* __restrict__ nm) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t i = (size_t)y * W + x;
    const float d = depth[i];
    const bool valid = d > 0.0f && isfinite(d);
    const float3 p = valid ? backproject((float)x, (float)y, d, fx, fy, cx, cy) : make_float3(0.0f, 0.0f, 0.0f);
    pm[3 * i + 0] = p.x;
    pm[3 * i + 1] = p.y;
    pm[3 * i + 2] = p.z;
    if (!nm) return;
    const float3 n = vsg::depth_normal(depth, W, H, x, y, fx, fy, cx, cy);
    nm[3 * i + 0] = n.x;
    nm[3 * i + 1] = n.y;
    nm[3 * i + 2] = n.z;
}

}  // namespace

extern "C" {

int vsg_depth_to_pointmap(const float* depth, int w, int h, float fx, float fy, float cx, float cy, float* pointmap,
                          float* normals, vsg_stream_t stream) {
    if (!depth || !pointmap || w <= 0 || h <= 0 || fx == 0.0f || fy == 0.0f) return VSG_ERR_INVALID_ARG;
    const dim3 grid((w + 31) / 32, (h + 7) / 8);
    k_depth_to_maps<<<grid, dim3(32, 8), 0, static_cast<cudaStream_t>(stream)>>>(depth, w, h, fx, fy, cx, cy,
                                                                                 pointmap, normals);
    return cudaGetLastError() == cudaSuccess ? VSG_OK : VSG_ERR_CUDA;
}

}  // extern "C"
