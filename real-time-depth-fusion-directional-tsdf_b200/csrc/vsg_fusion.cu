// vsg_fusion.cu -- block allocation, visible-block selection and TSDF
// integration kernels, plus the scene half of the C ABI (include/vsg.h).
//
// One frame is four stream-ordered launches and no host synchronisation:
//   k_frame_begin   clear the per-frame counters
//   k_alloc         per 16x16 pixel tile: DDA along each pixel's truncation
//                   band (VoxelScene.cu:295-633), de-duplicate the visited
//                   blocks in shared memory, insert the unique ones with a
//                   warp-cooperative atomicCAS bucket probe (8 lanes per
//                   key, one 128-B bucket line) and a linked-list overflow;
//                   also writes each pixel's world point T*p and camera
//                   distance once (bit-identical to the per-voxel
//                   recomputation of VoxelScene.cu:1052-1062)
//   k_select        visible-block compaction: one thread per pool block,
//                   conservative frustum + depth-band test (or new this
//                   frame), ballot + popc + one atomic per warp
//   k_integrate     persistent: one warp per visible block, 4 voxels per
//                   lane per batch with all gathers issued before use
//                   (VoxelScene.cu:918-1146)
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>

#include "../../include/vsg.h"
#include "vsg_device.cuh"
#include "vsg_fusion_core.cuh"
#include "vsg_internal.h"

namespace vsg {

// ====================================================================
// allocation
// ====================================================================

template <bool kByNormal>
__global__ void __launch_bounds__(kTile* kTile) k_alloc(AllocArgs a) {
    alloc_tile<kByNormal>(a, blockIdx.x, blockIdx.y);
}

__global__ void __launch_bounds__(256) k_parents(SceneDev s) {
    apply_parents(s, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

__global__ void __launch_bounds__(256) k_select(IntegArgs a) {
    select_blocks(a, blockIdx.x * blockDim.x, gridDim.x * blockDim.x);
}

// four resident CTAs per SM (<= 64 registers): more warps to cover the
// per-voxel divisions' latency (measured: 1280x720 / 2 mm frames 0.208 ms
// against 0.261 ms at two CTAs and 108 registers)
__global__ void __launch_bounds__(256, 4) k_integrate(IntegArgs a) { integrate_work(a); }

// ====================================================================
// scene management kernels
// ====================================================================

__global__ void k_init_heap(uint32_t* heap, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) heap[i] = (uint32_t)(n - 1 - i);  // initHeapKernel, VoxelScene.cu:250-255
}

__global__ void k_init_counters(SceneCounters* c, int num_blocks) {
    c->free_count = num_blocks;
    c->high_water = 0u;
    c->nodes_used = 0;
    c->flags = 0u;
    c->alloc_fail = 0u;
    c->coord_drops = 0u;
}

__global__ void k_frame_begin(FrameCounters* f) { frame_begin(f); }

// avg_div against IEEE division for every divisor d = 1..256 and every
// dividend x in [1, 2) (2^31 pairs; by the scaling argument at avg_div that
// covers 2^-100 <= |x| < 2^100): fail[d] = 1 where any quotient differs.
__global__ void k_verify_avg_div(unsigned int* fail) {
    const uint32_t n = 256u << 23;
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        const uint32_t d = (u >> 23) + 1u;
        const float x = __uint_as_float(0x3F800000u | (u & 0x7FFFFFu));
        const float df = (float)d;
        const float y = 1.0f / df;
        if (__float_as_uint(avg_div(x, df, y)) != __float_as_uint(x / df)) fail[d] = 1u;
    }
}

// ====================================================================
// host side
// ====================================================================

static size_t sup_words(int k) { return ((1ull << (3 * (k - 3))) + 31ull) / 32ull; }

// The running average's reciprocal table (SceneDev::avg_recip): RN(1/d) for
// the divisors that passed k_verify_avg_div, 0 for the others.  Which
// divisors pass is a property of IEEE binary32 arithmetic, not of a scene or
// a device, so it is verified once per process, on the GPU current at the
// first scene creation.
static int avg_recip_table(float out[257]) {
    static std::mutex mu;
    static bool done = false;
    static float table[257];
    std::lock_guard<std::mutex> lock(mu);
    if (!done) {
        unsigned int* fail = nullptr;
        if (cudaMalloc(&fail, 257 * sizeof(unsigned int)) != cudaSuccess) return VSG_ERR_OUT_OF_MEMORY;
        cudaMemset(fail, 0, 257 * sizeof(unsigned int));
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        k_verify_avg_div<<<sms * 8, 256>>>(fail);
        unsigned int h[257];
        const cudaError_t e = cudaMemcpy(h, fail, sizeof(h), cudaMemcpyDeviceToHost);
        cudaFree(fail);
        if (e != cudaSuccess) return VSG_ERR_CUDA;
        table[0] = 0.0f;
        for (int d = 1; d <= 256; ++d) table[d] = h[d] ? 0.0f : 1.0f / (float)d;
        done = true;
    }
    memcpy(out, table, sizeof(table));
    return VSG_OK;
}

int scene_alloc_device(Scene* sc) {
    SceneDev& d = sc->dev;
    const size_t S = sc->params.hash_num_slots, B = sc->params.num_sdf_blocks;
    const size_t M = sc->params.max_chain_nodes;
    cudaError_t e = cudaSuccess;
#define VSG_MALLOC(ptr, bytes)                                 \
    do {                                                       \
        e = cudaMalloc((void**)&(ptr), (bytes));               \
        if (e != cudaSuccess) return VSG_ERR_OUT_OF_MEMORY;    \
    } while (0)
    VSG_MALLOC(d.buckets, S * kBucketSlots * sizeof(Entry));
    VSG_MALLOC(d.bucket_next, S * sizeof(int));
    VSG_MALLOC(d.nodes, M * sizeof(Node));
    // one block more than the pool: block B stays all zero (weight 0) and
    // stands for "not allocated" in the ray caster's tap cache, so its tap
    // loads need no test
    VSG_MALLOC(d.voxels, (B + 1) * kVoxPerBlock * sizeof(Voxel));
    if (cudaMemset(d.voxels + B * kVoxPerBlock, 0, kVoxPerBlock * sizeof(Voxel)) != cudaSuccess) return VSG_ERR_CUDA;
    VSG_MALLOC(d.block_key, B * sizeof(unsigned long long));
    VSG_MALLOC(d.block_slot, B * sizeof(int));
    VSG_MALLOC(d.block_fresh, B);
    VSG_MALLOC(d.block_wmask, B * sizeof(unsigned long long));
    VSG_MALLOC(d.block_touched, B);
    VSG_MALLOC(d.block_parent, B * sizeof(unsigned long long));
    VSG_MALLOC(d.heap, B * sizeof(uint32_t));
    VSG_MALLOC(d.bindex, sizeof(unsigned long long) << (3 * sc->bidx_log2));
    VSG_MALLOC(d.dwm, sizeof(unsigned long long) << (3 * sc->bidx_log2));
    VSG_MALLOC(d.sup, sup_words(sc->bidx_log2) * 4);
    VSG_MALLOC(d.visible, B * sizeof(uint32_t));
    d.pix_world = nullptr;
    d.pix_rgb = nullptr;
    sc->pix_capacity = 0;
    d.parent_key = nullptr;
    d.parent_tag = nullptr;
    d.parent_cap = 0;
    d.alloc_method = 1;
    VSG_MALLOC(d.avg_recip, 257 * sizeof(float));
    VSG_MALLOC(d.ctr, sizeof(SceneCounters));
    VSG_MALLOC(d.frame, sizeof(FrameCounters));
#undef VSG_MALLOC
    d.num_buckets = (uint32_t)S;
    d.num_blocks = (int)B;
    d.max_nodes = (int)M;
    d.bidx_log2 = sc->bidx_log2;
    d.voxel = sc->params.voxel_size;
    d.inv_voxel = 1.0f / d.voxel;
    bool fast = false;
    if (verify_fixed_division(d.voxel, &fast) != VSG_OK) fast = false;
    d.div_fast = fast;
    {
        float tab[257];
        const int rc = avg_recip_table(tab);
        if (rc != VSG_OK) return rc;
        if (cudaMemcpy(const_cast<float*>(d.avg_recip), tab, sizeof(tab), cudaMemcpyHostToDevice) != cudaSuccess)
            return VSG_ERR_CUDA;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_integrate, 256, 0);
    sc->integ_ctas_per_sm = per_sm > 0 ? per_sm : 2;
    return VSG_OK;
}

void scene_free_device(Scene* sc) {
    SceneDev& d = sc->dev;
    void* ptrs[] = {d.block_parent, d.parent_key, d.parent_tag, d.block_touched, d.sup, d.dwm,     d.bindex,    d.block_wmask, d.buckets,   d.bucket_next,
                    d.nodes,     d.voxels,  d.block_key, d.block_slot,  d.block_fresh, d.heap,
                    d.visible,   d.pix_world, d.pix_rgb, d.ctr,         d.frame, const_cast<float*>(d.avg_recip)};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    memset(&d, 0, sizeof(d));
}

int scene_reset_device(Scene* sc, cudaStream_t st) {
    SceneDev& d = sc->dev;
    const size_t S = sc->params.hash_num_slots, B = sc->params.num_sdf_blocks;
    const size_t M = sc->params.max_chain_nodes;
    cudaMemsetAsync(d.buckets, 0xFF, S * kBucketSlots * sizeof(Entry), st);
    cudaMemsetAsync(d.bucket_next, 0xFF, S * sizeof(int), st);
    cudaMemsetAsync(d.nodes, 0xFF, M * sizeof(Node), st);
    cudaMemsetAsync(d.block_key, 0xFF, B * sizeof(unsigned long long), st);
    cudaMemsetAsync(d.block_fresh, 0, B, st);
    cudaMemsetAsync(d.block_parent, 0, B * sizeof(unsigned long long), st);
    cudaMemsetAsync(d.bindex, 0xFF, sizeof(unsigned long long) << (3 * sc->bidx_log2), st);
    cudaMemsetAsync(d.dwm, 0, sizeof(unsigned long long) << (3 * sc->bidx_log2), st);
    cudaMemsetAsync(d.sup, 0, sup_words(sc->bidx_log2) * 4, st);
    k_init_heap<<<(unsigned)((B + 255) / 256), 256, 0, st>>>(d.heap, (int)B);
    k_init_counters<<<1, 1, 0, st>>>(d.ctr, (int)B);
    k_frame_begin<<<1, 1, 0, st>>>(d.frame);
    sc->integrated_frames = 0;
    return cudaGetLastError() == cudaSuccess ? VSG_OK : VSG_ERR_CUDA;
}

// Parent records of one normal-direction allocation: a normal ray of length
// truncation visits at most 1 + 3 (floor(t / 8v) + 1) blocks; one record
// per (tile, block) and per block a full tile set could not take, so
// pixels x that bound covers every frame (grows only).
int ensure_parent_buffers(Scene* sc, size_t npx, float trunc) {
    SceneDev& d = sc->dev;
    const double ext = 8.0 * (double)d.voxel;
    const double per_ray = 1.0 + 3.0 * (std::floor(std::fabs((double)trunc) / ext) + 1.0);
    const double want = std::ceil((double)npx * per_ray);
    if (want > 4.0e9) return VSG_ERR_TOO_LARGE;
    if ((size_t)want <= d.parent_cap) return VSG_OK;
    cudaFree(d.parent_key);
    cudaFree(d.parent_tag);
    d.parent_key = nullptr;
    d.parent_tag = nullptr;
    d.parent_cap = 0;
    if (cudaMalloc(&d.parent_key, (size_t)want * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&d.parent_tag, (size_t)want * sizeof(uint32_t)) != cudaSuccess)
        return VSG_ERR_OUT_OF_MEMORY;
    d.parent_cap = (uint32_t)want;
    return VSG_OK;
}

int ensure_pixel_buffers(Scene* sc, size_t npx) {
    if (npx <= sc->pix_capacity) return VSG_OK;
    // grows only: a first frame of a larger resolution allocates (outside
    // any capture), later frames reuse
    cudaFree(sc->dev.pix_world);
    cudaFree(sc->dev.pix_rgb);
    sc->dev.pix_world = nullptr;
    sc->dev.pix_rgb = nullptr;
    sc->pix_capacity = 0;
    if (cudaMalloc(&sc->dev.pix_world, npx * sizeof(float4)) != cudaSuccess) return VSG_ERR_OUT_OF_MEMORY;
    if (cudaMalloc(&sc->dev.pix_rgb, npx * sizeof(uint32_t)) != cudaSuccess) return VSG_ERR_OUT_OF_MEMORY;
    sc->pix_capacity = npx;
    return VSG_OK;
}

int scene_integrate(Scene* sc, const float* pm, const uint8_t* rgb, const float* nm, int W, int H, float trunc,
                    const float* pose, float fx, float fy, float cx, float cy, cudaStream_t st) {
    const bool by_normal = sc->dev.alloc_method == 2;
    if (by_normal && (W > 65535 || H > 65535)) return VSG_ERR_TOO_LARGE;
    int prc = ensure_pixel_buffers(sc, (size_t)W * H);
    if (prc == VSG_OK && by_normal) prc = ensure_parent_buffers(sc, (size_t)W * H, trunc);
    if (prc != VSG_OK) return prc;
    sc->dev.frame_seq = sc->integrated_frames;
    Pose P;
    memcpy(P.T, pose, sizeof(P.T));
    k_frame_begin<<<1, 1, 0, st>>>(sc->dev.frame);
    AllocArgs aa;
    aa.s = sc->dev;
    aa.pm = pm;
    aa.rgb = rgb;
    aa.nm = nm;
    aa.W = W;
    aa.H = H;
    aa.trunc = trunc;
    aa.pose = P;
    dim3 grid((W + kTile - 1) / kTile, (H + kTile - 1) / kTile);
    timing_begin(sc, kSlotAlloc, st);
    if (by_normal) {
        k_alloc<true><<<grid, kTile * kTile, 0, st>>>(aa);
        k_parents<<<sc->sm_count * 2, 256, 0, st>>>(sc->dev);
    } else {
        k_alloc<false><<<grid, kTile * kTile, 0, st>>>(aa);
    }
    timing_end(sc, kSlotAlloc, st);
    IntegArgs ia;
    ia.s = sc->dev;
    ia.W = W;
    ia.H = H;
    ia.trunc = trunc;
    ia.pose = P;
    ia.fx = fx;
    ia.fy = fy;
    ia.cx = cx;
    ia.cy = cy;
    timing_begin(sc, kSlotSelect, st);
    k_select<<<sc->sm_count * 4, 256, 0, st>>>(ia);
    timing_end(sc, kSlotSelect, st);
    timing_begin(sc, kSlotIntegrate, st);
    k_integrate<<<sc->sm_count * sc->integ_ctas_per_sm, 256, 0, st>>>(ia);
    timing_end(sc, kSlotIntegrate, st);
    sc->integrated_frames++;
    return cudaGetLastError() == cudaSuccess ? VSG_OK : VSG_ERR_CUDA;
}

// Same launch sequence as scene_integrate, with the per-pixel work buffers
// supplied by the caller (at least W*H entries each) instead of the scene's
// own, and without event timing; allocates nothing.
int scene_integrate_with_pixels(Scene* sc, const float* pm, const uint8_t* rgb, int W, int H, float trunc,
                                const float* pose, float fx, float fy, float cx, float cy, float4* pix_world,
                                uint32_t* pix_rgb, cudaStream_t st) {
    // normal-direction allocation keeps per-frame parent records in buffers
    // of the scene's own: not available here
    if (sc->dev.alloc_method == 2) return VSG_ERR_INVALID_ARG;
    Pose P;
    memcpy(P.T, pose, sizeof(P.T));
    SceneDev dev = sc->dev;
    dev.pix_world = pix_world;
    dev.pix_rgb = pix_rgb;
    k_frame_begin<<<1, 1, 0, st>>>(dev.frame);
    AllocArgs aa;
    aa.s = dev;
    aa.pm = pm;
    aa.rgb = rgb;
    aa.nm = nullptr;
    aa.W = W;
    aa.H = H;
    aa.trunc = trunc;
    aa.pose = P;
    dim3 grid((W + kTile - 1) / kTile, (H + kTile - 1) / kTile);
    k_alloc<false><<<grid, kTile * kTile, 0, st>>>(aa);
    IntegArgs ia;
    ia.s = dev;
    ia.W = W;
    ia.H = H;
    ia.trunc = trunc;
    ia.pose = P;
    ia.fx = fx;
    ia.fy = fy;
    ia.cx = cx;
    ia.cy = cy;
    k_select<<<sc->sm_count * 4, 256, 0, st>>>(ia);
    k_integrate<<<sc->sm_count * sc->integ_ctas_per_sm, 256, 0, st>>>(ia);
    sc->integrated_frames++;
    return cudaGetLastError() == cudaSuccess ? VSG_OK : VSG_ERR_CUDA;
}

}  // namespace vsg
