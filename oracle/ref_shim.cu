// ref_shim.cu -- TEST INFRASTRUCTURE ONLY.
//
// A plain C interface over the reference's own CUDA launchers so the checker
// can run them: compiled by oracle/ref_build.py together with the
// reference's VoxelScene.cu, RayCastRender.cu, CUDAHashRef.cu and
// MarchingCubes.cu (from their own source tree) into oracle/_ref/.  It
// mirrors what VoxelScene::integrateFromScanData (VoxelScene.cpp:404-833)
// and main's ray-cast block (voxelSG.cpp:575-618) do, minus the logging and
// file dumps, and reads the hash table back in a neutral format.  The
// product never loads this.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "CUDAHashRef.h"
#include "MarchingCubes.h"
#include "VoxelScene.h"

extern "C" void rayCastRenderCUDA(CUDAHashRef& hashData, int width, int height, float* d_depth, float4* d_depth4,
                                  float4* d_colors, float4* d_normals, float3 cameraPos, float* cameraTransform,
                                  float fx, float fy, float cx, float cy, float minDepth, float maxDepth,
                                  float voxelSize, int numBuckets, int bucketSize, int totalHashSize);

extern "C" void extractSurfacePointsCUDA(const CUDAHashRef& hashData, const Params& params, float minSDF,
                                         float maxSDF, unsigned int minWeight, float4* d_outputPositions,
                                         float4* d_outputColors, float4* d_outputNormals, int maxPoints,
                                         int* d_pointCount);

namespace {
struct RefScene {
    CUDAHashRef hash;
    Params params;
};
}  // namespace

extern "C" {

void* ref_create(int slots, int blocks, float voxel, float trunc, float trunc_scale) {
    RefScene* s = new RefScene();
    Params& p = s->params;
    p.hashSlotNum = slots;  // CUDAHashData.h:14-29
    p.SDFBlockNum = blocks;
    p.SDFBlockSize = SDF_BLOCK_SIZE;
    p.slotSize = HASH_BUCKET_SIZE;
    p.totalHashSize = slots * HASH_BUCKET_SIZE;
    p.totalBlockSize = blocks * SDF_BLOCK_SIZE * SDF_BLOCK_SIZE * SDF_BLOCK_SIZE;
    p.voxelSize = voxel;
    p.truncationScale = trunc;
    p.truncation = trunc_scale;
    s->hash.HashDataAllocation(p);
    resetHashDataCUDA(s->hash, p);
    return s;
}

void ref_destroy(void* h) {
    RefScene* s = static_cast<RefScene*>(h);
    if (!s) return;
    CUDAHashRef& d = s->hash;
    void* ptrs[] = {d.d_hashTable, d.d_CompactifiedHashTable, d.d_hashCompactifiedCounter, d.d_SDFBlocks,
                    d.d_blockParentUV, d.d_blockAllocationMethod, d.d_hashBucketMutex, d.d_heap, d.d_heapCounter,
                    d.d_voxelZeroCross, d.d_voxelZeroCrossCounter, d.d_hashDecision, d.d_hashDecisionPrefix};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete s;
}

// integrateFromScanData without logging: device pose copy, camera position =
// translation column (VoxelScene.cpp:431-466), allocate, compact, integrate.
int ref_integrate(void* h, const float* pm, const uint8_t* rgb, const float* nm, int W, int H, float trunc,
                  const float* T_host, float fx, float fy, float cx, float cy) {
    RefScene* s = static_cast<RefScene*>(h);
    float* d_T = nullptr;
    if (cudaMalloc(&d_T, 16 * sizeof(float)) != cudaSuccess) return 1;
    cudaMemcpy(d_T, T_host, 16 * sizeof(float), cudaMemcpyHostToDevice);
    const float3 cam = make_float3(T_host[3], T_host[7], T_host[11]);
    allocBlocksFromDepthMapCUDA(s->hash, s->params, reinterpret_cast<const float3*>(pm),
                                reinterpret_cast<const float3*>(nm), W, H, trunc, cam, d_T);
    compactifyHashCUDA(s->hash, s->params);
    integrateDepthMapIntoBlocksCUDA(s->hash, s->params, reinterpret_cast<const float3*>(pm),
                                    reinterpret_cast<const uchar3*>(rgb), reinterpret_cast<const float3*>(nm), W, H,
                                    trunc, cam, d_T, fx, fy, cx, cy);
    cudaFree(d_T);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

// The same with the reference's normal-direction allocation, as its build
// with USE_NORMAL_DIR_ALLOC calls it (VoxelScene.cu:1693-1715).
int ref_integrate_m2(void* h, const float* pm, const uint8_t* rgb, const float* nm, int W, int H, float trunc,
                     const float* T_host, float fx, float fy, float cx, float cy) {
    RefScene* s = static_cast<RefScene*>(h);
    float* d_T = nullptr;
    if (cudaMalloc(&d_T, 16 * sizeof(float)) != cudaSuccess) return 1;
    cudaMemcpy(d_T, T_host, 16 * sizeof(float), cudaMemcpyHostToDevice);
    const float3 cam = make_float3(T_host[3], T_host[7], T_host[11]);
    allocBlocksFromDepthMapMethod2CUDA(s->hash, s->params, reinterpret_cast<const float3*>(pm),
                                       reinterpret_cast<const float3*>(nm), W, H, trunc, cam, d_T);
    compactifyHashCUDA(s->hash, s->params);
    integrateDepthMapIntoBlocksCUDA(s->hash, s->params, reinterpret_cast<const float3*>(pm),
                                    reinterpret_cast<const uchar3*>(rgb), reinterpret_cast<const float3*>(nm), W, H,
                                    trunc, cam, d_T, fx, fy, cx, cy);
    cudaFree(d_T);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

// RayCastRender::extractSurfacePoints without its logging
// (RayCastRender.cpp:307-368): the points to host float4 arrays of max_pts
// entries.  Returns the reference's point count (or -1).
int ref_extract_points(void* h, float min_sdf, float max_sdf, unsigned int min_w, int max_pts, float* pos,
                       float* col, float* nrm) {
    RefScene* s = static_cast<RefScene*>(h);
    float4 *dp = nullptr, *dc = nullptr, *dn = nullptr;
    int* dcnt = nullptr;
    if (cudaMalloc(&dp, (size_t)max_pts * sizeof(float4)) != cudaSuccess ||
        cudaMalloc(&dc, (size_t)max_pts * sizeof(float4)) != cudaSuccess ||
        cudaMalloc(&dn, (size_t)max_pts * sizeof(float4)) != cudaSuccess || cudaMalloc(&dcnt, sizeof(int)) != cudaSuccess)
        return -1;
    extractSurfacePointsCUDA(s->hash, s->params, min_sdf, max_sdf, min_w, dp, dc, dn, max_pts, dcnt);
    int n = -1;
    cudaMemcpy(&n, dcnt, sizeof(int), cudaMemcpyDeviceToHost);
    const int k = n < 0 ? 0 : (n < max_pts ? n : max_pts);
    cudaMemcpy(pos, dp, (size_t)k * sizeof(float4), cudaMemcpyDeviceToHost);
    cudaMemcpy(col, dc, (size_t)k * sizeof(float4), cudaMemcpyDeviceToHost);
    cudaMemcpy(nrm, dn, (size_t)k * sizeof(float4), cudaMemcpyDeviceToHost);
    cudaFree(dp);
    cudaFree(dc);
    cudaFree(dn);
    cudaFree(dcnt);
    return cudaDeviceSynchronize() == cudaSuccess ? n : -1;
}

// main's ray-cast block (voxelSG.cpp:575-618): outputs to host buffers
// (depth float[W*H], position / colour / normal float4[W*H]).
int ref_render(void* h, int W, int H, const float* T_host, float fx, float fy, float cx, float cy, float minD,
               float maxD, float* depth, float* pos, float* col, float* nrm) {
    RefScene* s = static_cast<RefScene*>(h);
    const size_t n = (size_t)W * H;
    float* d_depth = nullptr;
    float4 *d_pos = nullptr, *d_col = nullptr, *d_nrm = nullptr;
    float* d_T = nullptr;
    cudaMalloc(&d_depth, n * sizeof(float));
    cudaMalloc(&d_pos, n * sizeof(float4));
    cudaMalloc(&d_col, n * sizeof(float4));
    cudaMalloc(&d_nrm, n * sizeof(float4));
    cudaMalloc(&d_T, 16 * sizeof(float));
    // fill the outputs with the caller's contents (the reference leaves them
    // untouched when the scene is empty)
    cudaMemcpy(d_depth, depth, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_pos, pos, n * sizeof(float4), cudaMemcpyHostToDevice);
    cudaMemcpy(d_col, col, n * sizeof(float4), cudaMemcpyHostToDevice);
    cudaMemcpy(d_nrm, nrm, n * sizeof(float4), cudaMemcpyHostToDevice);
    cudaMemcpy(d_T, T_host, 16 * sizeof(float), cudaMemcpyHostToDevice);
    const float3 cam = make_float3(T_host[3], T_host[7], T_host[11]);
    rayCastRenderCUDA(s->hash, W, H, d_depth, d_pos, d_col, d_nrm, cam, d_T, fx, fy, cx, cy, minD, maxD,
                      s->params.voxelSize, s->params.hashSlotNum, s->params.slotSize, s->params.totalHashSize);
    cudaMemcpy(depth, d_depth, n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemcpy(pos, d_pos, n * sizeof(float4), cudaMemcpyDeviceToHost);
    cudaMemcpy(col, d_col, n * sizeof(float4), cudaMemcpyDeviceToHost);
    cudaMemcpy(nrm, d_nrm, n * sizeof(float4), cudaMemcpyDeviceToHost);
    cudaFree(d_depth);
    cudaFree(d_pos);
    cudaFree(d_col);
    cudaFree(d_nrm);
    cudaFree(d_T);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

// Allocated blocks: coords int32[n*3] (hash order) and 512 voxels each as
// 8-byte records (float sdf, uint8 r, g, b, weight).  Returns n, or -1 when
// more than max_blocks are allocated.
int ref_export(void* h, int32_t* coords, uint8_t* vox8, int max_blocks) {
    RefScene* s = static_cast<RefScene*>(h);
    const size_t E = (size_t)s->params.totalHashSize;
    std::vector<HashSlot> table(E);
    cudaMemcpy(table.data(), s->hash.d_hashTable, E * sizeof(HashSlot), cudaMemcpyDeviceToHost);
    int n = 0;
    std::vector<VoxelData> blk(512);
    for (size_t i = 0; i < E; ++i) {
        if (table[i].ptr == -1) continue;
        if (n >= max_blocks) return -1;
        coords[3 * n + 0] = table[i].pos.x;
        coords[3 * n + 1] = table[i].pos.y;
        coords[3 * n + 2] = table[i].pos.z;
        if (vox8) {
            cudaMemcpy(blk.data(), s->hash.d_SDFBlocks + (size_t)table[i].ptr * 512, 512 * sizeof(VoxelData),
                       cudaMemcpyDeviceToHost);
            for (int v = 0; v < 512; ++v) {
                uint8_t* o = vox8 + ((size_t)n * 512 + v) * 8;
                std::memcpy(o, &blk[v].sdf, 4);
                o[4] = blk[v].color.x;
                o[5] = blk[v].color.y;
                o[6] = blk[v].color.z;
                o[7] = blk[v].weight;
            }
        }
        ++n;
    }
    return n;
}

int ref_voxel_bytes(void) { return (int)sizeof(VoxelData); }

// Device-resident variants for timing the reference's launchers: inputs,
// outputs and the pose already on the device; the returned value is the
// device time (ms, CUDA events) of the launcher calls, host work inside them
// (their own syncs and small allocations) included.
float ref_integrate_dev(void* h, const float* pm, const uint8_t* rgb, const float* nm, int W, int H, float trunc,
                        const float* T_host, float* T_dev, float fx, float fy, float cx, float cy) {
    RefScene* s = static_cast<RefScene*>(h);
    const float3 cam = make_float3(T_host[3], T_host[7], T_host[11]);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    allocBlocksFromDepthMapCUDA(s->hash, s->params, reinterpret_cast<const float3*>(pm),
                                reinterpret_cast<const float3*>(nm), W, H, trunc, cam, T_dev);
    compactifyHashCUDA(s->hash, s->params);
    integrateDepthMapIntoBlocksCUDA(s->hash, s->params, reinterpret_cast<const float3*>(pm),
                                    reinterpret_cast<const uchar3*>(rgb), reinterpret_cast<const float3*>(nm), W, H,
                                    trunc, cam, T_dev, fx, fy, cx, cy);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = -1.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return cudaDeviceSynchronize() == cudaSuccess ? ms : -1.0f;
}

float ref_render_dev(void* h, int W, int H, const float* T_host, float* T_dev, float fx, float fy, float cx, float cy,
                     float minD, float maxD, float* depth, float* pos, float* col, float* nrm) {
    RefScene* s = static_cast<RefScene*>(h);
    const float3 cam = make_float3(T_host[3], T_host[7], T_host[11]);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    rayCastRenderCUDA(s->hash, W, H, depth, reinterpret_cast<float4*>(pos), reinterpret_cast<float4*>(col),
                      reinterpret_cast<float4*>(nrm), cam, T_dev, fx, fy, cx, cy, minD, maxD, s->params.voxelSize,
                      s->params.hashSlotNum, s->params.slotSize, s->params.totalHashSize);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = -1.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return cudaDeviceSynchronize() == cudaSuccess ? ms : -1.0f;
}

}  // extern "C"
