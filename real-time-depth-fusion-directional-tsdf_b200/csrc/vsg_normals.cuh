// vsg_normals.cuh -- the depth-image normal fallback of
// CustomDepthMapGenerator (CustomDepthMapGenerator.cpp:163-209), shared by
// the depth -> point-map converter and the point-cloud splat.
#pragma once

#include <cuda_runtime.h>

namespace vsg {

// (x - cx) d / fx, (y - cy) d / fy, d: the generator's back-projection.
__device__ __forceinline__ float3 backproject(float x, float y, float d, float fx, float fy, float cx, float cy) {
    return make_float3((x - cx) * d / fx, (y - cy) * d / fy, d);
}

// Normal of pixel (x, y) of a W x H depth image: for interior pixels with
// depth > 0 the normalised cross product of (right - centre) and (down -
// centre), back-projected from the three depths as stored (an invalid
// neighbour's 0 included); (0,0,0) elsewhere and for a zero-length cross.
__device__ __forceinline__ float3 depth_normal(const float* __restrict__ depth, int W, int H, int x, int y, float fx,
                                               float fy, float cx, float cy) {
    float3 n = make_float3(0.0f, 0.0f, 0.0f);
    const size_t i = (size_t)y * W + x;
    const float d = depth[i];
    if (x >= 1 && x < W - 1 && y >= 1 && y < H - 1 && d > 0.0f) {
        const float dr = depth[i + 1], dd = depth[i + W];
        const float3 c = backproject((float)x, (float)y, d, fx, fy, cx, cy);
        const float3 r = backproject((float)(x + 1), (float)y, dr, fx, fy, cx, cy);
        const float3 w = backproject((float)x, (float)(y + 1), dd, fx, fy, cx, cy);
        const float ax = r.x - c.x, ay = r.y - c.y, az = r.z - c.z;
        const float bx = w.x - c.x, by = w.y - c.y, bz = w.z - c.z;
        const float3 cr = make_float3(ay * bz - az * by, az * bx - ax * bz, ax * by - ay * bx);
        const float len = sqrtf(cr.x * cr.x + cr.y * cr.y + cr.z * cr.z);
        if (len > 0.0f) {
            const float inv = 1.0f / len;
            n = make_float3(cr.x * inv, cr.y * inv, cr.z * inv);
        }
    }
    return n;
}

}  // namespace vsg
