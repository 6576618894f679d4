// vsg_mc.cu -- marching cubes over the scene's voxel blocks.
//
// Restates marchingCubesKernel / runMarchingCubesCUDA (MarchingCubes.cu:
// 352-467, 508-571): every allocated block, every cube whose eight voxels lie
// inside the block (local x, y, z < 7, :379), corners at (8b + v + 0.5) *
// voxel, case bit k set when corner k's SDF is below the iso value (weights
// are not read), edge vertices by vertexInterp (:313-327), one face normal per
// triangle by computeNormal (:329-350), triangles appended through one
// counter.  The case table (vsg_mc_table.h) holds the reference's triangle
// rows for its 186 well-formed cases, entry for entry, and generated rows for
// the 70 cases its table leaves undefined (rows missing past 208, rows 140,
// 184-186, 189 and 191-208 naming edges their case does not cross).
//
// Layout of the work: one CTA of 352 threads walks the pool blocks; per
// block it stages the 512 SDF values in shared memory, gives each of the 343
// cubes one thread, scans the per-cube triangle counts across the CTA and
// reserves the block's range of the output with ONE atomic, then every
// thread writes its triangles.  Blocks with no weighted voxel hold SDF 0
// everywhere (fresh blocks are zeroed and a voxel's SDF changes only with its
// weight), so every cube of such a block has the same case (0 or 255) and no
// triangle: they are skipped on their weight mask without reading voxels.
#include <cuda_runtime.h>

#include <climits>
#include <new>

#include "../../include/vsg.h"
#include "vsg_device.cuh"
#include "vsg_internal.h"
#include "vsg_mc_table.h"

namespace vsg {
namespace {

constexpr int kMcThreads = 352;  // 11 warps; cube i = thread i (7^3 = 343)
constexpr int kMcWarps = kMcThreads / 32;

struct McCounters {
    unsigned long long total;  // triangles of the surface (may exceed the capacity)
    int total_i32;             // min(total, INT_MAX): the reference's int counter
    int pad;
};

__device__ __forceinline__ int corner_dx(int k) { return (k ^ (k >> 1)) & 1; }
__device__ __forceinline__ int corner_dy(int k) { return (k >> 1) & 1; }
__device__ __forceinline__ int corner_dz(int k) { return k >> 2; }

// edge e -> its first and second corner (kMcEdge): edges 0-3 and 4-7 run
// around the z=0 and z=1 faces, edges 8-11 join corner e-8 to corner e-4
__device__ __forceinline__ int edge_c0(int e) { return e < 8 ? e : e - 8; }
__device__ __forceinline__ int edge_c1(int e) { return e < 8 ? ((e & 4) | ((e + 1) & 3)) : e - 4; }

__global__ void __launch_bounds__(kMcThreads) k_marching_cubes(SceneDev s, const uint4* __restrict__ table,
                                                               float iso, float voxel, float* __restrict__ verts,
                                                               float* __restrict__ norms, McCounters* ctr,
                                                               int max_tris) {
    __shared__ float sdf[kVoxPerBlock];
    __shared__ __align__(16) unsigned char tab[256 * 16];
    __shared__ int warp_tot[kMcWarps];
    __shared__ unsigned long long s_base;
    for (int i = threadIdx.x; i < 256; i += kMcThreads) reinterpret_cast<uint4*>(tab)[i] = table[i];

    const uint32_t hw = s.ctr->high_water;
    const int cube = threadIdx.x;
    const int lx = cube % 7, ly = (cube / 7) % 7, lz = cube / 49;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float extent = (float)kBlock * voxel;  // MarchingCubes.cu:384

    for (uint32_t b = blockIdx.x; b < hw; b += gridDim.x) {
        const unsigned long long key = s.block_key[b];
        if (key == kKeyEmpty || key == kKeyTomb) continue;
        if (s.block_fresh[b] || s.block_wmask[b] == 0ull) continue;
        __syncthreads();  // table staged; previous block's readers done
        const Voxel* vb = s.voxels + (size_t)b * kVoxPerBlock;
        for (int i = threadIdx.x; i < kVoxPerBlock; i += kMcThreads) sdf[i] = vb[i].sdf;
        __syncthreads();

        int ci = 0, ntri = 0;
        if (cube < 343) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int v = ((lz + corner_dz(k)) * kBlock + ly + corner_dy(k)) * kBlock + lx + corner_dx(k);
                if (sdf[v] < iso) ci |= 1 << k;  // :407-415
            }
            ntri = (ci == 0 || ci == 255) ? 0 : tab[ci * 16 + 15];
        }
        // CTA-wide exclusive scan of the per-cube triangle counts
        int incl = ntri;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        int before = 0, total = 0;
#pragma unroll
        for (int w = 0; w < kMcWarps; ++w) {
            const int t = warp_tot[w];
            before += w < warp ? t : 0;
            total += t;
        }
        if (threadIdx.x == 0) {
            unsigned long long base = 0ull;
            if (total) {
                base = atomicAdd(&ctr->total, (unsigned long long)total);
                const unsigned long long end = base + (unsigned long long)total;
                atomicMax(&ctr->total_i32, end > (unsigned long long)INT_MAX ? INT_MAX : (int)end);
            }
            s_base = base;
        }
        __syncthreads();
        if (ntri == 0) continue;

        int bx, by, bz;
        unpack_key(key, bx, by, bz);
        const float base_x = (float)bx * extent, base_y = (float)by * extent, base_z = (float)bz * extent;
        const unsigned long long first = s_base + (unsigned long long)(before + incl - ntri);
        const unsigned char* row = tab + ci * 16;
        for (int t = 0; t < ntri; ++t) {
            const unsigned long long o = first + (unsigned long long)t;
            if (o >= (unsigned long long)max_tris) break;
            float p[3][3];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const int e = row[3 * t + j];
                const int c0 = edge_c0(e), c1 = edge_c1(e);
                const int ax = lx + corner_dx(c0), ay = ly + corner_dy(c0), az = lz + corner_dz(c0);
                const int bx1 = lx + corner_dx(c1), by1 = ly + corner_dy(c1), bz1 = lz + corner_dz(c1);
                const float v1 = sdf[(az * kBlock + ay) * kBlock + ax];
                const float v2 = sdf[(bz1 * kBlock + by1) * kBlock + bx1];
                // cornerPos, :401-404
                const float p1x = base_x + ((float)ax + 0.5f) * voxel;
                const float p1y = base_y + ((float)ay + 0.5f) * voxel;
                const float p1z = base_z + ((float)az + 0.5f) * voxel;
                const float p2x = base_x + ((float)bx1 + 0.5f) * voxel;
                const float p2y = base_y + ((float)by1 + 0.5f) * voxel;
                const float p2z = base_z + ((float)bz1 + 0.5f) * voxel;
                // vertexInterp, :313-327
                const float denom = v2 - v1;
                if (fabsf(denom) < 1e-6f) {
                    p[j][0] = 0.5f * (p1x + p2x);
                    p[j][1] = 0.5f * (p1y + p2y);
                    p[j][2] = 0.5f * (p1z + p2z);
                } else {
                    float mu = __fdiv_rn(iso - v1, denom);
                    mu = fminf(fmaxf(mu, 0.0f), 1.0f);
                    p[j][0] = p1x + mu * (p2x - p1x);
                    p[j][1] = p1y + mu * (p2y - p1y);
                    p[j][2] = p1z + mu * (p2z - p1z);
                }
            }
            // computeNormal, :329-350
            const float ax = p[1][0] - p[0][0], ay = p[1][1] - p[0][1], az = p[1][2] - p[0][2];
            const float bxx = p[2][0] - p[0][0], byy = p[2][1] - p[0][1], bzz = p[2][2] - p[0][2];
            float nx = ay * bzz - az * byy;
            float ny = az * bxx - ax * bzz;
            float nz = ax * byy - ay * bxx;
            const float len = __fsqrt_rn(nx * nx + ny * ny + nz * nz);
            if (len > 1e-6f) {
                const float inv = __fdiv_rn(1.0f, len);
                nx *= inv;
                ny *= inv;
                nz *= inv;
            } else {
                nx = ny = nz = 0.0f;
            }
            float* ov = verts + o * 9;
            float* on = norms + o * 9;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                ov[3 * j + 0] = p[j][0];
                ov[3 * j + 1] = p[j][1];
                ov[3 * j + 2] = p[j][2];
                on[3 * j + 0] = nx;
                on[3 * j + 1] = ny;
                on[3 * j + 2] = nz;
            }
        }
    }
}

}  // namespace

struct McOutput {
    float* vertices = nullptr;  // float3[3 * max_tris]
    float* normals = nullptr;   // float3[3 * max_tris]
    McCounters* ctr = nullptr;
    uint4* table = nullptr;     // 256 x 16 bytes
    int max_tris = 0;
    int device = 0;
};

}  // namespace vsg

struct vsg_mc_output {
    vsg::McOutput impl;
};

namespace {

const unsigned char* host_table() {
    static unsigned char tab[256][16];
    static const bool built = (vsg_mc_build_table(tab), true);
    (void)built;
    return &tab[0][0];
}

}  // namespace

extern "C" {

int vsg_mc_output_create(int max_triangles, vsg_mc_output** out) {
    if (!out || max_triangles <= 0) return VSG_ERR_INVALID_ARG;
    *out = nullptr;
    vsg_mc_output* m = new (std::nothrow) vsg_mc_output();
    if (!m) return VSG_ERR_OUT_OF_MEMORY;
    vsg::McOutput& o = m->impl;
    cudaGetDevice(&o.device);
    const size_t bytes = (size_t)max_triangles * 9 * sizeof(float);
    if (cudaMalloc(&o.vertices, bytes) != cudaSuccess || cudaMalloc(&o.normals, bytes) != cudaSuccess ||
        cudaMalloc(&o.ctr, sizeof(vsg::McCounters)) != cudaSuccess || cudaMalloc(&o.table, 256 * 16) != cudaSuccess) {
        cudaFree(o.vertices);
        cudaFree(o.normals);
        cudaFree(o.ctr);
        cudaFree(o.table);
        delete m;
        return VSG_ERR_OUT_OF_MEMORY;
    }
    if (cudaMemcpy(o.table, host_table(), 256 * 16, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(o.ctr, 0, sizeof(vsg::McCounters)) != cudaSuccess) {
        cudaFree(o.vertices);
        cudaFree(o.normals);
        cudaFree(o.ctr);
        cudaFree(o.table);
        delete m;
        return VSG_ERR_CUDA;
    }
    o.max_tris = max_triangles;
    *out = m;
    return VSG_OK;
}

int vsg_mc_output_destroy(vsg_mc_output* m) {
    if (!m) return VSG_ERR_INVALID_ARG;
    cudaFree(m->impl.vertices);
    cudaFree(m->impl.normals);
    cudaFree(m->impl.ctr);
    cudaFree(m->impl.table);
    delete m;
    return VSG_OK;
}

int vsg_mc_run(vsg_scene* s, vsg_mc_output* m, float iso, float voxel_size, vsg_stream_t stream) {
    if (!s || !m) return VSG_ERR_INVALID_ARG;
    vsg::Scene* sc = &s->impl;
    vsg::McOutput& o = m->impl;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != sc->device || dev != o.device) return VSG_ERR_INVALID_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // paramsMC.voxelSize > 0 ? paramsMC.voxelSize : params.voxelSize (MarchingCubes.cu:543)
    const float voxel = voxel_size > 0.0f ? voxel_size : sc->params.voxel_size;
    if (cudaMemsetAsync(o.ctr, 0, sizeof(vsg::McCounters), st) != cudaSuccess) return VSG_ERR_CUDA;
    vsg::timing_begin(sc, vsg::kSlotMarchingCubes, st);
    const int grid = sc->sm_count * 4;
    vsg::k_marching_cubes<<<grid, vsg::kMcThreads, 0, st>>>(sc->dev, o.table, iso, voxel, o.vertices, o.normals,
                                                            o.ctr, o.max_tris);
    vsg::timing_end(sc, vsg::kSlotMarchingCubes, st);
    return cudaGetLastError() == cudaSuccess ? VSG_OK : VSG_ERR_CUDA;
}

int vsg_mc_triangle_count(const vsg_mc_output* m, int64_t* count) {
    if (!m || !count) return VSG_ERR_INVALID_ARG;
    int dev = -1;  // the synchronisation below waits for the current device only
    if (cudaGetDevice(&dev) != cudaSuccess || dev != m->impl.device) return VSG_ERR_INVALID_ARG;
    if (cudaDeviceSynchronize() != cudaSuccess) return VSG_ERR_CUDA;
    vsg::McCounters c{};
    if (cudaMemcpy(&c, m->impl.ctr, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess) return VSG_ERR_CUDA;
    *count = (int64_t)c.total;
    return VSG_OK;
}

int vsg_mc_output_buffers(const vsg_mc_output* m, float** vertices, float** normals, int** count_dev,
                          int* max_triangles) {
    if (!m) return VSG_ERR_INVALID_ARG;
    if (vertices) *vertices = m->impl.vertices;
    if (normals) *normals = m->impl.normals;
    if (count_dev) *count_dev = &m->impl.ctr->total_i32;
    if (max_triangles) *max_triangles = m->impl.max_tris;
    return VSG_OK;
}

int vsg_mc_download(const vsg_mc_output* m, float* vertices, float* normals, int64_t* count) {
    if (!m) return VSG_ERR_INVALID_ARG;
    int64_t n = 0;
    const int rc = vsg_mc_triangle_count(m, &n);
    if (rc != VSG_OK) return rc;
    if (count) *count = n;
    const size_t bytes = (size_t)(n < m->impl.max_tris ? n : m->impl.max_tris) * 9 * sizeof(float);
    if (bytes && vertices && cudaMemcpy(vertices, m->impl.vertices, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        return VSG_ERR_CUDA;
    if (bytes && normals && cudaMemcpy(normals, m->impl.normals, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        return VSG_ERR_CUDA;
    return VSG_OK;
}

}  // extern "C"
