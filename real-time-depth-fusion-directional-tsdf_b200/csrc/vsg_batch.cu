// vsg_batch.cu -- many independent scenes advanced together.
//
// A batched step integrates (and optionally ray casts) one frame for each of
// up to kMaxBatch scenes of any resolution with ONE launch per stage for all
// of them: the per-scene work is addressed through argument blocks uploaded
// in a single copy, and CTAs find their scene from prefix sums of per-scene
// tile counts.  The launch sequence of a step is captured into a CUDA graph
// and replayed while the batch's shape (which scenes, their resolutions)
// stays the same; only the argument blocks change.  Each stage runs exactly
// the per-scene device code (vsg_fusion_core.cuh, vsg_raycast_core.cuh), so
// every scene's results are identical to vsg_integrate + vsg_render.
//
// Autotuning: the ray-cast stage exists in five register budgets (CTAs per
// SM 4 to 8); vsg_batch_step with autotune on times each on the step's own
// data (ray casting does not modify the scene, so repeating it is harmless)
// and keeps the fastest for the batch's shape.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "../../include/vsg.h"
#include "vsg_device.cuh"
#include "vsg_fusion_core.cuh"
#include "vsg_internal.h"
#include "vsg_raycast_core.cuh"

namespace vsg {

constexpr int kMaxBatch = 256;
constexpr int kRenderTileW = 16, kRenderTileH = 8;

struct BatchHeader {
    int n;
    int pad[3];
    uint32_t alloc_prefix[kMaxBatch + 1];   // 16x16 allocation tiles before scene i
    uint32_t render_prefix[kMaxBatch + 1];  // 16x8 ray-cast tiles before scene i
    int alloc_tiles_x[kMaxBatch];
    int render_tiles_x[kMaxBatch];
};

// device layout of one step: header, then n AllocArgs, IntegArgs, RenderArgs
struct BatchLayout {
    size_t alloc_off, integ_off, render_off, bytes;
};

static BatchLayout layout_for(int n) {
    auto up = [](size_t v) { return (v + 255) & ~size_t(255); };
    BatchLayout L;
    L.alloc_off = up(sizeof(BatchHeader));
    L.integ_off = up(L.alloc_off + sizeof(AllocArgs) * n);
    L.render_off = up(L.integ_off + sizeof(IntegArgs) * n);
    L.bytes = up(L.render_off + sizeof(RenderArgs) * n);
    return L;
}

__device__ __forceinline__ int scene_of(const uint32_t* prefix, int n, uint32_t t) {
    int lo = 0, hi = n - 1;  // largest i with prefix[i] <= t
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void k_batch_frame_begin(const BatchHeader* h, const IntegArgs* integ) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < h->n) frame_begin(integ[i].s.frame);
}

__global__ void __launch_bounds__(kTile* kTile) k_batch_alloc(const BatchHeader* h, const AllocArgs* args) {
    const int i = scene_of(h->alloc_prefix, h->n, blockIdx.x);
    const uint32_t t = blockIdx.x - h->alloc_prefix[i];
    alloc_tile<false>(args[i], (int)(t % (uint32_t)h->alloc_tiles_x[i]), (int)(t / (uint32_t)h->alloc_tiles_x[i]));
}

__global__ void __launch_bounds__(256) k_batch_select(const BatchHeader* h, const IntegArgs* args) {
    if ((int)blockIdx.y >= h->n) return;
    select_blocks(args[blockIdx.y], blockIdx.x * blockDim.x, gridDim.x * blockDim.x);
}

// Integration of every scene's visible blocks as one work queue: a prefix of
// the scenes' visible counts (written by the selection), then every warp of
// the launch takes the next (scene, visible block) from one counter, so no
// scene's blocks wait on a fixed share of the GPU while other scenes' share
// sits idle.  Each visible block is integrated by exactly one warp, as in
// integrate_work.
__global__ void k_batch_visible_prefix(const BatchHeader* h, const IntegArgs* args, uint32_t* queue) {
    if (threadIdx.x != 0) return;
    uint32_t s = 0;
    for (int i = 0; i < h->n; ++i) {
        queue[i] = s;
        s += *(volatile uint32_t*)&args[i].s.frame->n_visible;
    }
    queue[h->n] = s;
    queue[kMaxBatch + 1] = 0u;  // the work counter
}

__global__ void __launch_bounds__(256, 4) k_batch_integrate(const BatchHeader* h, const IntegArgs* args,
                                                           uint32_t* queue) {
    const int lane = threadIdx.x & 31;
    const uint32_t total = queue[h->n];
    for (;;) {
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(queue + kMaxBatch + 1, 1u);
        g = __shfl_sync(0xFFFFFFFFu, g, 0);
        if (g >= total) break;
        const int i = scene_of(queue, h->n, g);
        const IntegArgs& a = args[i];
        const uint32_t b = a.s.visible[g - queue[i]];
        integrate_block(a, (int)b, a.s.block_key[b], a.s.block_fresh[b] != 0, lane);
    }
}

// The ray-distance bounds of every scene ray cast this step: cleared, then
// filled by tile_bounds_range over each scene's pool blocks.
__global__ void __launch_bounds__(256) k_batch_bounds_clear(const BatchHeader* h, const RenderArgs* args) {
    if ((int)blockIdx.y >= h->n) return;
    const RenderArgs& a = args[blockIdx.y];
    if (a.W <= 0 || !a.bounds) return;
    uint2* b = const_cast<uint2*>(a.bounds);
    const int n = a.n1 + a.n2 + 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = make_uint2(0u, 0u);
}

__global__ void __launch_bounds__(256) k_batch_tile_bounds(const BatchHeader* h, const RenderArgs* args) {
    if ((int)blockIdx.y >= h->n) return;
    const RenderArgs& a = args[blockIdx.y];
    if (a.W <= 0 || !a.bounds) return;
    tile_bounds_range(a, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// The ray-cast tiles of every scene of the step in one order, longest march
// range first (tile_bucket), as for one scene (k_tile_hist, k_tile_scatter)
// over the tiles' step-wide indices.  The grid covers the largest step
// (all renderers); counts (16 counts, 16 cursors) is zeroed before.
__global__ void __launch_bounds__(256) k_batch_tile_hist(const BatchHeader* h, const RenderArgs* args,
                                                         unsigned* counts) {
    __shared__ unsigned hist[kOrderBuckets];
    if (threadIdx.x < kOrderBuckets) hist[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < h->render_prefix[h->n]) {
        const int i = scene_of(h->render_prefix, h->n, g);
        const uint32_t t = g - h->render_prefix[i], tx = (uint32_t)h->render_tiles_x[i];
        atomicAdd(&hist[tile_bucket(args[i], (int)(t % tx), (int)(t / tx))], 1u);
    }
    __syncthreads();
    if (threadIdx.x < kOrderBuckets && hist[threadIdx.x]) atomicAdd(counts + threadIdx.x, hist[threadIdx.x]);
}

__global__ void __launch_bounds__(256) k_batch_tile_scatter(const BatchHeader* h, const RenderArgs* args,
                                                            uint32_t* order, unsigned* counts) {
    __shared__ unsigned start[kOrderBuckets];
    if (threadIdx.x == 0) {
        unsigned s = 0;
        for (int b = kOrderBuckets - 1; b >= 0; --b) {  // heaviest bucket first
            start[b] = s;
            s += counts[b];
        }
    }
    __syncthreads();
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < h->render_prefix[h->n]) {
        const int i = scene_of(h->render_prefix, h->n, g);
        const uint32_t t = g - h->render_prefix[i], tx = (uint32_t)h->render_tiles_x[i];
        const int b = tile_bucket(args[i], (int)(t % tx), (int)(t / tx));
        order[start[b] + atomicAdd(counts + kOrderBuckets + b, 1u)] = g;
    }
}

template <int kMinBlocks>
__global__ void __launch_bounds__(128, kMinBlocks) k_batch_render(const BatchHeader* h, const RenderArgs* args,
                                                                  const uint32_t* __restrict__ order) {
    const uint32_t g = __ldg(order + blockIdx.x);
    const int i = scene_of(h->render_prefix, h->n, g);
    const RenderArgs& a = args[i];
    if (a.W <= 0) return;  // scene not ray cast this step
    const uint32_t t = g - h->render_prefix[i];
    const int tx = (int)(t % (uint32_t)h->render_tiles_x[i]), ty = (int)(t / (uint32_t)h->render_tiles_x[i]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = tx * kRenderTileW + (warp & 1) * 8 + (lane & 7);
    const int y = ty * kRenderTileH + (warp >> 1) * 4 + (lane >> 3);
    if (x >= a.W || y >= a.H) return;
    render_pixel<false>(a, x, y);
}

struct Batch {
    int device = 0;
    int sm_count = 148;
    std::vector<Scene*> scenes;
    std::vector<Renderer*> renderers;
    unsigned char* d_step = nullptr;     // device copy of the step's argument blocks
    uint32_t* d_order = nullptr;         // ray-cast tile order of a step, then 32 counters
    uint32_t* d_queue = nullptr;         // integration queue: visible-count prefix, then the work counter
    int integ_ctas_per_sm = 4;           // resident CTAs of k_batch_integrate
    uint32_t order_cap = 0;              // ray-cast tiles of all renderers together
    unsigned char* h_step[2] = {};       // pinned staging, alternate steps
    cudaEvent_t done[2] = {};            // last step that read h_step[i] finished
    bool pending[2] = {false, false};
    int parity = 0;
    size_t step_bytes = 0;
    bool autotune = true;
    struct Shape {
        cudaGraphExec_t exec[2] = {nullptr, nullptr};  // one per staging buffer
        int render_variant = -1;  // 0: 6 CTAs/SM, 1: 4, 2: 8, 3: 5, 4: 7; -1 = not tuned yet
    };
    std::map<std::vector<int>, Shape> shapes;
};

static void launch_render_variant(int v, dim3 grid, cudaStream_t st, const BatchHeader* h, const RenderArgs* r,
                                  const uint32_t* order) {
    if (v == 1)
        k_batch_render<4><<<grid, 128, 0, st>>>(h, r, order);
    else if (v == 2)
        k_batch_render<8><<<grid, 128, 0, st>>>(h, r, order);
    else if (v == 3)
        k_batch_render<5><<<grid, 128, 0, st>>>(h, r, order);
    else if (v == 4)
        k_batch_render<7><<<grid, 128, 0, st>>>(h, r, order);
    else
        k_batch_render<6><<<grid, 128, 0, st>>>(h, r, order);
}

}  // namespace vsg

struct vsg_batch {
    vsg::Batch impl;
};

using vsg::Batch;

namespace vsg {

// Enqueue the ray-distance bounds of the scenes a step ray casts.
static void enqueue_bounds(Batch& b, int n, cudaStream_t st) {
    const BatchLayout L = layout_for(n);
    const BatchHeader* h = reinterpret_cast<const BatchHeader*>(b.d_step);
    const RenderArgs* ra = reinterpret_cast<const RenderArgs*>(b.d_step + L.render_off);
    const int bnd_x = std::max(2, (b.sm_count * 4) / n);
    k_batch_bounds_clear<<<dim3(bnd_x, n), 256, 0, st>>>(h, ra);
    k_batch_tile_bounds<<<dim3(bnd_x, n), 256, 0, st>>>(h, ra);
    unsigned* counts = b.d_order + b.order_cap;
    const unsigned grid = std::max(1u, (b.order_cap + 255) / 256);
    cudaMemsetAsync(counts, 0, 2 * kOrderBuckets * sizeof(unsigned), st);
    k_batch_tile_hist<<<grid, 256, 0, st>>>(h, ra, counts);
    k_batch_tile_scatter<<<grid, 256, 0, st>>>(h, ra, b.d_order, counts);
}

// Enqueue the stages of one step (argument blocks already on the device).
static void enqueue_stages(Batch& b, int n, uint32_t alloc_tiles, uint32_t render_tiles, int render_variant,
                           cudaStream_t st) {
    const BatchLayout L = layout_for(n);
    const BatchHeader* h = reinterpret_cast<const BatchHeader*>(b.d_step);
    const AllocArgs* aa = reinterpret_cast<const AllocArgs*>(b.d_step + L.alloc_off);
    const IntegArgs* ia = reinterpret_cast<const IntegArgs*>(b.d_step + L.integ_off);
    const RenderArgs* ra = reinterpret_cast<const RenderArgs*>(b.d_step + L.render_off);
    k_batch_frame_begin<<<(n + 127) / 128, 128, 0, st>>>(h, ia);
    if (alloc_tiles) k_batch_alloc<<<alloc_tiles, kTile * kTile, 0, st>>>(h, aa);
    const int sel_x = std::max(2, (b.sm_count * 8) / n);
    k_batch_select<<<dim3(sel_x, n), 256, 0, st>>>(h, ia);
    k_batch_visible_prefix<<<1, 32, 0, st>>>(h, ia, b.d_queue);
    k_batch_integrate<<<b.sm_count * b.integ_ctas_per_sm, 256, 0, st>>>(h, ia, b.d_queue);
    if (render_tiles) {
        enqueue_bounds(b, n, st);
        launch_render_variant(render_variant, dim3(render_tiles), st, h, ra, b.d_order);
    }
}

}  // namespace vsg

extern "C" {

int vsg_batch_create(vsg_scene* const* scenes, vsg_renderer* const* renderers, int n, vsg_batch** out) {
    return vsg::host_guard([&]() -> int {
        if (!out || !scenes || n <= 0) return VSG_ERR_INVALID_ARG;
        if (n > vsg::kMaxBatch) return VSG_ERR_TOO_LARGE;
        *out = nullptr;
        vsg_batch* b = new (std::nothrow) vsg_batch();
        if (!b) return VSG_ERR_OUT_OF_MEMORY;
        Batch& B = b->impl;
        cudaGetDevice(&B.device);
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, B.device);
        B.sm_count = sms > 0 ? sms : 148;
        for (int i = 0; i < n; ++i) {
            if (!scenes[i] || scenes[i]->impl.device != B.device) {
                delete b;
                return VSG_ERR_INVALID_ARG;
            }
            if (renderers && renderers[i] && renderers[i]->impl.device != B.device) {
                delete b;
                return VSG_ERR_INVALID_ARG;
            }
            B.scenes.push_back(&scenes[i]->impl);
            B.renderers.push_back(renderers ? (renderers[i] ? &renderers[i]->impl : nullptr) : nullptr);
        }
        for (const vsg::Renderer* r : B.renderers)
            if (r) B.order_cap += (uint32_t)(((r->w + vsg::kRenderTileW - 1) / vsg::kRenderTileW) *
                                             ((r->h + vsg::kRenderTileH - 1) / vsg::kRenderTileH));
        B.step_bytes = vsg::layout_for(vsg::kMaxBatch).bytes;
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vsg::k_batch_integrate, 256, 0);
        B.integ_ctas_per_sm = per_sm > 0 ? per_sm : 4;
        bool ok = cudaMalloc(&B.d_step, B.step_bytes) == cudaSuccess &&
                  cudaMalloc(&B.d_order, sizeof(uint32_t) * (B.order_cap + 32)) == cudaSuccess &&
                  cudaMalloc(&B.d_queue, sizeof(uint32_t) * (vsg::kMaxBatch + 2)) == cudaSuccess;
        for (int i = 0; i < 2 && ok; ++i)
            ok = cudaMallocHost(&B.h_step[i], B.step_bytes) == cudaSuccess &&
                 cudaEventCreateWithFlags(&B.done[i], cudaEventDisableTiming) == cudaSuccess;
        if (!ok) {
            cudaFree(B.d_step);
            cudaFree(B.d_order);
            cudaFree(B.d_queue);
            for (int i = 0; i < 2; ++i) {
                if (B.h_step[i]) cudaFreeHost(B.h_step[i]);
                if (B.done[i]) cudaEventDestroy(B.done[i]);
            }
            delete b;
            return VSG_ERR_OUT_OF_MEMORY;
        }
        for (int i = 0; i < 2; ++i) memset(B.h_step[i], 0, B.step_bytes);
        *out = b;
        return VSG_OK;
    });
}

int vsg_batch_destroy(vsg_batch* b) {
    if (!b) return VSG_ERR_INVALID_ARG;
    cudaDeviceSynchronize();
    for (auto& kv : b->impl.shapes)
        for (int i = 0; i < 2; ++i)
            if (kv.second.exec[i]) cudaGraphExecDestroy(kv.second.exec[i]);
    cudaFree(b->impl.d_step);
    cudaFree(b->impl.d_order);
    cudaFree(b->impl.d_queue);
    for (int i = 0; i < 2; ++i) {
        cudaFreeHost(b->impl.h_step[i]);
        cudaEventDestroy(b->impl.done[i]);
    }
    delete b;
    return VSG_OK;
}

int vsg_batch_autotune(vsg_batch* b, int enable) {
    if (!b) return VSG_ERR_INVALID_ARG;
    b->impl.autotune = enable != 0;
    return VSG_OK;
}

int vsg_batch_step(vsg_batch* b, const vsg_batch_frame* frames, int n_frames, vsg_stream_t stream) {
    return vsg::host_guard([&]() -> int {
        using namespace vsg;
        if (!b) return VSG_ERR_NOT_ALLOCATED;
        if (!frames || n_frames <= 0) return VSG_ERR_INVALID_ARG;
        Batch& B = b->impl;
        if (n_frames > (int)B.scenes.size()) return VSG_ERR_INVALID_ARG;
        cudaStream_t st = (cudaStream_t)stream;
        int dev = -1;
        if (cudaGetDevice(&dev) != cudaSuccess || dev != B.device) return VSG_ERR_INVALID_ARG;
        // validate, make sure each scene's per-pixel buffers fit (allocates only
        // on a scene's first frame of a larger resolution)
        std::vector<char> seen(B.scenes.size(), 0);
        for (int k = 0; k < n_frames; ++k) {
            const vsg_batch_frame& f = frames[k];
            if (f.scene < 0 || f.scene >= (int)B.scenes.size() || seen[f.scene]) return VSG_ERR_INVALID_ARG;
            seen[f.scene] = 1;
            if (!f.pointmap || !f.rgb || !f.normals || f.w <= 0 || f.h <= 0) return VSG_ERR_INVALID_ARG;
            // normal-direction allocation needs its own parent pass: per-scene calls only
            if (B.scenes[f.scene]->dev.alloc_method == 2) return VSG_ERR_INVALID_ARG;
            if (f.render) {
                Renderer* r = B.renderers[f.scene];
                if (!r || r->w != f.w || r->h != f.h) return VSG_ERR_INVALID_ARG;
            }
            const int rc = ensure_pixel_buffers(B.scenes[f.scene], (size_t)f.w * f.h);
            if (rc != VSG_OK) return rc;
        }
        // alternate staging buffers; the step that last read this one must be done
        const int pb = B.parity;
        B.parity ^= 1;
        if (B.pending[pb]) {
            cudaEventSynchronize(B.done[pb]);
            B.pending[pb] = false;
        }
        unsigned char* hs = B.h_step[pb];
        const BatchLayout L = layout_for(n_frames);
        BatchHeader* h = reinterpret_cast<BatchHeader*>(hs);
        AllocArgs* aa = reinterpret_cast<AllocArgs*>(hs + L.alloc_off);
        IntegArgs* ia = reinterpret_cast<IntegArgs*>(hs + L.integ_off);
        RenderArgs* ra = reinterpret_cast<RenderArgs*>(hs + L.render_off);
        h->n = n_frames;
        std::vector<int> key;
        key.push_back(n_frames);
        uint32_t at = 0, rt = 0;
        for (int k = 0; k < n_frames; ++k) {
            const vsg_batch_frame& f = frames[k];
            Scene* sc = B.scenes[f.scene];
            const int ax = (f.w + kTile - 1) / kTile, ay = (f.h + kTile - 1) / kTile;
            h->alloc_prefix[k] = at;
            h->alloc_tiles_x[k] = ax;
            at += (uint32_t)(ax * ay);
            const int rx = (f.w + kRenderTileW - 1) / kRenderTileW, ry = (f.h + kRenderTileH - 1) / kRenderTileH;
            h->render_prefix[k] = rt;
            h->render_tiles_x[k] = rx;
            if (f.render) rt += (uint32_t)(rx * ry);
            key.push_back(f.w);
            key.push_back(f.h);
            key.push_back(f.render ? 1 : 0);
            Pose P;
            memcpy(P.T, f.pose, sizeof(P.T));
            AllocArgs& A = aa[k];
            A.s = sc->dev;
            A.pm = f.pointmap;
            A.rgb = f.rgb;
            A.nm = f.normals;
            A.W = f.w;
            A.H = f.h;
            A.trunc = f.truncation;
            A.pose = P;
            IntegArgs& I = ia[k];
            I.s = sc->dev;
            I.W = f.w;
            I.H = f.h;
            I.trunc = f.truncation;
            I.pose = P;
            I.fx = f.fx;
            I.fy = f.fy;
            I.cx = f.cx;
            I.cy = f.cy;
            RenderArgs& R = ra[k];
            memset(&R, 0, sizeof(R));
            R.s = sc->dev;
            if (f.render) {
                Renderer* r = B.renderers[f.scene];
                R.W = f.w;
                R.H = f.h;
                R.camx = f.pose[3];
                R.camy = f.pose[7];
                R.camz = f.pose[11];
                R.pose = P;
                R.pose_dev = nullptr;
                R.touched = nullptr;
                R.fx = f.fx;
                R.fy = f.fy;
                R.cx = f.cx;
                R.cy = f.cy;
                R.minD = f.min_depth;
                R.maxD = f.max_depth;
                R.step = r->step;
                R.depth = r->depth;
                R.pos = r->position;
                R.col = r->color;
                R.nrm = r->normal;
                // the renderer's bounds buffer (sized for r->w x r->h == f.w x f.h)
                R.bounds = r->bounds;
                R.t1x = (f.w + 7) / 8;
                R.t2x = (f.w + 63) / 64;
                R.n1 = R.t1x * ((f.h + 3) / 4);
                R.n2 = R.t2x * ((f.h + 31) / 32);
            }
            sc->integrated_frames++;
        }
        h->alloc_prefix[n_frames] = at;
        h->render_prefix[n_frames] = rt;
        const size_t bytes = L.bytes;
        Batch::Shape& shape = B.shapes[key];
        if (shape.render_variant < 0) {
            // first step of this shape: run it eagerly, tuning the ray-cast
            // variant on the step's own data (ray casting leaves the scene as it
            // is, so repeating it only rewrites the same outputs)
            if (cudaMemcpyAsync(B.d_step, hs, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) return VSG_ERR_CUDA;
            enqueue_stages(B, n_frames, at, 0, 0, st);
            int best = 0;
            if (rt) {
                enqueue_bounds(B, n_frames, st);
                const BatchHeader* dh = reinterpret_cast<const BatchHeader*>(B.d_step);
                const RenderArgs* dr = reinterpret_cast<const RenderArgs*>(B.d_step + L.render_off);
                if (B.autotune) {
                    float best_ms = 3.4e38f;
                    cudaEvent_t e0, e1;
                    cudaEventCreate(&e0);
                    cudaEventCreate(&e1);
                    for (int v = 0; v < 5; ++v) {
                        cudaEventRecord(e0, st);
                        launch_render_variant(v, dim3(rt), st, dh, dr, B.d_order);
                        cudaEventRecord(e1, st);
                        cudaEventSynchronize(e1);
                        float ms = 0.0f;
                        cudaEventElapsedTime(&ms, e0, e1);
                        if (ms < best_ms) {
                            best_ms = ms;
                            best = v;
                        }
                    }
                    cudaEventDestroy(e0);
                    cudaEventDestroy(e1);
                } else {
                    launch_render_variant(0, dim3(rt), st, dh, dr, B.d_order);
                }
            }
            shape.render_variant = best;
            cudaEventRecord(B.done[pb], st);
            B.pending[pb] = true;
            // capture the step for replay: copy of the argument blocks from
            // staging buffer i, then the stages; one graph per staging buffer
            for (int i = 0; i < 2; ++i) {
                cudaStream_t cs;
                if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return VSG_ERR_CUDA;
                cudaGraph_t g = nullptr;
                cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
                cudaMemcpyAsync(B.d_step, B.h_step[i], bytes, cudaMemcpyHostToDevice, cs);
                enqueue_stages(B, n_frames, at, rt, best, cs);
                const cudaError_t ce = cudaStreamEndCapture(cs, &g);
                cudaStreamDestroy(cs);
                if (ce != cudaSuccess || !g) return VSG_ERR_CUDA;
                const cudaError_t ie = cudaGraphInstantiate(&shape.exec[i], g, 0);
                cudaGraphDestroy(g);
                if (ie != cudaSuccess) {
                    shape.exec[i] = nullptr;
                    return VSG_ERR_CUDA;
                }
            }
            return cudaGetLastError() == cudaSuccess ? VSG_OK : VSG_ERR_CUDA;
        }
        if (cudaGraphLaunch(shape.exec[pb], st) != cudaSuccess) return VSG_ERR_CUDA;
        cudaEventRecord(B.done[pb], st);
        B.pending[pb] = true;
        return cudaGetLastError() == cudaSuccess ? VSG_OK : VSG_ERR_CUDA;
    });
}

}  // extern "C"
