// vsg_batch.cu -- many independent scenes advanced together in one
// persistent launch.
//
// A batched step integrates (and optionally ray casts) one frame for each of
// up to kMaxBatch scenes of any resolution with ONE launch of k_batch_step.
// Its CTAs -- as many as fit on the GPU at once -- take work items from a
// device counter, in a fixed stage-major order:
//   stage 0  per scene: clear its frame counters and ray-distance bounds
//   stage 1  allocation tiles, 16x16 pixels (alloc_tile)
//   stage 2  visible-block selection, strided over the pool (select_blocks)
//   stage 3  integration workers, each taking visible blocks from the
//            scene's work counter (integrate_work)
//   stage 4  ray-distance bounds, strided over the pool (tile_bounds_range)
//   stage 5  ray-cast workers: each warp takes 8x4 pixel tiles from the
//            scene's tile counter until none is left (render_pixel), so a
//            CTA waits for its slowest warp once per item, not per tile
// An item of stage k of scene i first waits until every item of the scene's
// previous non-empty stage has finished: per scene and stage a counter that
// finished items raise (release: CTA barrier, fence, atomic add) and that a
// waiting CTA polls with acquire loads.  So one scene's ray cast starts as
// soon as its own bounds are done, while other scenes still integrate, and
// no stage waits for the slowest scene of the previous stage.  Items are
// claimed in order, so an item only ever waits for items claimed earlier by
// CTAs that are running; the earliest unfinished item never waits, and the
// launch always completes.  Each wait is bounded all the same: after
// kWaitLimit polls the item records VSG_FLAG_BATCH_WAIT in the scene's flags,
// raises the launch's abort word -- every later wait of the launch then
// returns at once, so a launch stalls for at most about one wait limit --
// and goes on.  Data written earlier in the same launch (pixel buffers,
// hash, voxels, skip grids, bounds) is read through the coherent load path
// (VSG_COHERENT_LOADS).  Each stage runs exactly the per-scene device code
// (vsg_fusion_core.cuh, vsg_raycast_core.cuh), so every scene's results are
// identical to vsg_integrate + vsg_render.
//
// The step's launch (the copy of its argument blocks, the reset of the item
// and stage counters, k_batch_step) is captured into a CUDA graph and
// replayed while the batch's shape (which scenes, their resolutions) stays
// the same; only the argument blocks change.
//
// Autotuning: the number of resident CTAs per SM of k_batch_step.  On the
// first step of a shape, with autotune on, ray-cast-only launches of the
// same step (stage 0 clearing the bounds, stages 4 and 5; repeating them
// rewrites the same outputs) are timed at each candidate and the fastest is
// kept for the shape.
#define VSG_COHERENT_LOADS 1

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
constexpr int kStages = 6;
constexpr int kStepThreads = 256;
constexpr int kTilesPerWarp = 6;  // ray-cast workers per scene: 8x4 tiles / (8 warps x this)
constexpr int kWaitLimit = 1 << 22;  // polls of 64-128 ns: about a second
// claim counter and abort word (own line), stage counters, ray-cast tile counters
constexpr int kSyncWords = 32 + kMaxBatch * kStages + kMaxBatch;

struct BatchHeader {
    int n;
    int full;         // 1: the whole step; 0: ray cast only (stage 0 clears bounds only; stages 4, 5)
    uint32_t n_items;
    uint32_t pad;
    uint32_t stage_end[kStages];               // items of stages 0..s, all scenes
    uint32_t prefix[kStages][kMaxBatch + 1];   // items of stage s of the scenes before i
    int alloc_tiles_x[kMaxBatch];
};

// device layout of one step: the header of the whole step, the header of its
// ray-cast-only form, then n AllocArgs, IntegArgs, RenderArgs
struct BatchLayout {
    size_t render_hdr_off, alloc_off, integ_off, render_off, bytes;
};

static BatchLayout layout_for(int n) {
    auto up = [](size_t v) { return (v + 255) & ~size_t(255); };
    BatchLayout L;
    L.render_hdr_off = up(sizeof(BatchHeader));
    L.alloc_off = up(L.render_hdr_off + sizeof(BatchHeader));
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

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Whole CTA: wait until *ctr reaches `target`.  Bounded: after kWaitLimit
// polls flag the scene, raise the launch's abort word and go on; once the
// abort word is up no wait of the launch polls any more.
__device__ __forceinline__ void wait_stage(const uint32_t* ctr, uint32_t target, uint32_t* scene_flags,
                                           uint32_t* abort_word) {
    if (threadIdx.x == 0 && target) {
        int polls = 0;
        while (ld_acquire_u32(ctr) < target) {
            if (*(volatile uint32_t*)abort_word) break;
            if (++polls > kWaitLimit) {
                atomicOr(scene_flags, (uint32_t)VSG_FLAG_BATCH_WAIT);
                atomicExch(abort_word, 1u);
                break;
            }
            __nanosleep(64);
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kStepThreads, 3) k_batch_step(const BatchHeader* __restrict__ h,
                                                                const AllocArgs* __restrict__ aa,
                                                                const IntegArgs* __restrict__ ia,
                                                                const RenderArgs* __restrict__ ra, uint32_t* sync) {
    __shared__ uint32_t s_item;
    uint32_t* claim = sync;
    uint32_t* abort_word = sync + 1;
    uint32_t* done = sync + 32;
    uint32_t* tiles = done + kMaxBatch * kStages;
    const int n = h->n;
    const uint32_t total = h->n_items;
    const int lane = threadIdx.x & 31;
    for (;;) {
        __syncthreads();  // every thread has read the previous s_item
        if (threadIdx.x == 0) s_item = atomicAdd(claim, 1u);
        __syncthreads();
        const uint32_t g = s_item;
        if (g >= total) return;
        int st = 0;
        while (st < kStages - 1 && g >= h->stage_end[st]) ++st;
        const uint32_t t = g - (st ? h->stage_end[st - 1] : 0u);
        const int i = scene_of(h->prefix[st], n, t);
        const uint32_t k = t - h->prefix[st][i];
        const uint32_t cnt = h->prefix[st][i + 1] - h->prefix[st][i];
        if (st > 0) {
            int prev = st - 1;
            while (prev > 0 && h->prefix[prev][i + 1] == h->prefix[prev][i]) --prev;
            wait_stage(done + i * kStages + prev, h->prefix[prev][i + 1] - h->prefix[prev][i],
                       &ia[i].s.ctr->flags, abort_word);
        }
        if (st == 0) {
            if (h->full && threadIdx.x == 0) frame_begin(ia[i].s.frame);
            const RenderArgs& R = ra[i];
            if (R.W > 0 && R.bounds) {
                uint2* b = const_cast<uint2*>(R.bounds);
                const int nb = R.n1 + R.n2 + 1;
                for (int j = threadIdx.x; j < nb; j += kStepThreads) b[j] = make_uint2(0u, 0u);
            }
        } else if (st == 1) {
            const int tx = h->alloc_tiles_x[i];
            alloc_tile<false>(aa[i], (int)(k % (uint32_t)tx), (int)(k / (uint32_t)tx));
        } else if (st == 2) {
            select_blocks(ia[i], k * kStepThreads, cnt * kStepThreads);
        } else if (st == 3) {
            integrate_work(ia[i]);
        } else if (st == 4) {
            tile_bounds_range(ra[i], k * kStepThreads + threadIdx.x, cnt * kStepThreads);
        } else {
            const RenderArgs& R = ra[i];
            const int tx = (R.W + 7) / 8;
            const uint32_t ntiles = (uint32_t)tx * (uint32_t)((R.H + 3) / 4);
            for (;;) {
                uint32_t tt = 0;
                if (lane == 0) tt = atomicAdd(tiles + i, 1u);
                tt = __shfl_sync(0xFFFFFFFFu, tt, 0);
                if (tt >= ntiles) break;
                const int x = (int)(tt % (uint32_t)tx) * 8 + (lane & 7), y = (int)(tt / (uint32_t)tx) * 4 + (lane >> 3);
                if (x < R.W && y < R.H) render_pixel(R, x, y);
            }
        }
        __syncthreads();  // the item's writes are done
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(done + i * kStages + st, 1u);
        }
    }
}

struct Batch {
    int device = 0;
    int sm_count = 148;
    int max_ctas_per_sm = 1;             // occupancy of k_batch_step
    std::vector<Scene*> scenes;
    std::vector<Renderer*> renderers;
    unsigned char* d_step = nullptr;     // device copy of the step's argument blocks
    uint32_t* d_sync = nullptr;          // item and stage counters of the running step
    unsigned char* h_step[2] = {};       // pinned staging, alternate steps
    cudaEvent_t done[2] = {};            // last step that read h_step[i] finished
    bool pending[2] = {false, false};
    int parity = 0;
    size_t step_bytes = 0;
    bool autotune = true;
    struct Shape {
        cudaGraphExec_t exec[2] = {nullptr, nullptr};  // one per staging buffer
        int ctas_per_sm = -1;  // resident CTAs per SM of the launch; -1 = not tuned yet
    };
    std::map<std::vector<int>, Shape> shapes;
};

}  // namespace vsg

struct vsg_batch {
    vsg::Batch impl;
};

using vsg::Batch;

namespace vsg {

// Enqueue one launch of the step whose argument blocks are on the device:
// reset the counters, then k_batch_step with the given header.
static void enqueue_step(Batch& b, int n, bool render_only, int ctas_per_sm, cudaStream_t st) {
    const BatchLayout L = layout_for(n);
    const BatchHeader* h = reinterpret_cast<const BatchHeader*>(b.d_step + (render_only ? L.render_hdr_off : 0));
    const AllocArgs* aa = reinterpret_cast<const AllocArgs*>(b.d_step + L.alloc_off);
    const IntegArgs* ia = reinterpret_cast<const IntegArgs*>(b.d_step + L.integ_off);
    const RenderArgs* ra = reinterpret_cast<const RenderArgs*>(b.d_step + L.render_off);
    cudaMemsetAsync(b.d_sync, 0, sizeof(uint32_t) * kSyncWords, st);
    k_batch_step<<<b.sm_count * std::max(1, std::min(ctas_per_sm, b.max_ctas_per_sm)), kStepThreads, 0, st>>>(
        h, aa, ia, ra, b.d_sync);
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
            B.scenes.push_back(&scenes[i]->impl);
            B.renderers.push_back(renderers ? (renderers[i] ? &renderers[i]->impl : nullptr) : nullptr);
        }
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, vsg::k_batch_step, vsg::kStepThreads, 0);
        B.max_ctas_per_sm = occ > 0 ? occ : 1;
        B.step_bytes = vsg::layout_for(vsg::kMaxBatch).bytes;
        bool ok = cudaMalloc(&B.d_step, B.step_bytes) == cudaSuccess &&
                  cudaMalloc(&B.d_sync, sizeof(uint32_t) * vsg::kSyncWords) == cudaSuccess;
        for (int i = 0; i < 2 && ok; ++i)
            ok = cudaMallocHost(&B.h_step[i], B.step_bytes) == cudaSuccess &&
                 cudaEventCreateWithFlags(&B.done[i], cudaEventDisableTiming) == cudaSuccess;
        if (!ok) {
            cudaFree(B.d_step);
            cudaFree(B.d_sync);
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
    cudaFree(b->impl.d_sync);
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
        BatchHeader* hr = reinterpret_cast<BatchHeader*>(hs + L.render_hdr_off);
        AllocArgs* aa = reinterpret_cast<AllocArgs*>(hs + L.alloc_off);
        IntegArgs* ia = reinterpret_cast<IntegArgs*>(hs + L.integ_off);
        RenderArgs* ra = reinterpret_cast<RenderArgs*>(hs + L.render_off);
        // items per scene and stage (stage-major order); pool-strided stages
        // and the integration workers spread the GPU over the step's scenes
        const int sel_items = std::max(2, (B.sm_count * 8) / n_frames);
        const int integ_items = std::max(2, (B.sm_count * 4) / n_frames);
        const int bnd_items = std::max(2, (B.sm_count * 4) / n_frames);
        h->n = hr->n = n_frames;
        h->full = 1;
        hr->full = 0;
        std::vector<int> key;
        key.push_back(n_frames);
        uint32_t cnt[kStages][kMaxBatch];
        uint32_t cnt_r[kStages][kMaxBatch];
        bool any_render = false;
        for (int k = 0; k < n_frames; ++k) {
            const vsg_batch_frame& f = frames[k];
            Scene* sc = B.scenes[f.scene];
            const int ax = (f.w + kTile - 1) / kTile, ay = (f.h + kTile - 1) / kTile;
            const int rtiles = ((f.w + 7) / 8) * ((f.h + 3) / 4);
            const int rworkers = std::max(1, (rtiles + kStepThreads / 32 * kTilesPerWarp - 1) /
                                                 (kStepThreads / 32 * kTilesPerWarp));
            h->alloc_tiles_x[k] = hr->alloc_tiles_x[k] = ax;
            cnt[0][k] = 1;
            cnt[1][k] = (uint32_t)(ax * ay);
            cnt[2][k] = (uint32_t)sel_items;
            cnt[3][k] = (uint32_t)integ_items;
            cnt[4][k] = f.render ? (uint32_t)bnd_items : 0u;
            cnt[5][k] = f.render ? (uint32_t)rworkers : 0u;
            cnt_r[0][k] = f.render ? 1u : 0u;
            cnt_r[1][k] = cnt_r[2][k] = cnt_r[3][k] = 0u;
            cnt_r[4][k] = cnt[4][k];
            cnt_r[5][k] = cnt[5][k];
            any_render |= f.render != 0;
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
        uint32_t all = 0, all_r = 0;
        for (int st = 0; st < kStages; ++st) {
            uint32_t a = 0, b = 0;
            for (int k = 0; k < n_frames; ++k) {
                h->prefix[st][k] = a;
                hr->prefix[st][k] = b;
                a += cnt[st][k];
                b += cnt_r[st][k];
            }
            h->prefix[st][n_frames] = a;
            hr->prefix[st][n_frames] = b;
            all += a;
            all_r += b;
            h->stage_end[st] = all;
            hr->stage_end[st] = all_r;
        }
        h->n_items = all;
        hr->n_items = all_r;
        const size_t bytes = L.bytes;
        Batch::Shape& shape = B.shapes[key];
        if (shape.ctas_per_sm < 0) {
            // first step of this shape: run it eagerly, then time ray-cast-only
            // launches of it (they rewrite the same outputs) at each resident
            // CTA count, keep the fastest, and capture the step for replay
            if (cudaMemcpyAsync(B.d_step, hs, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) return VSG_ERR_CUDA;
            enqueue_step(B, n_frames, false, B.max_ctas_per_sm, st);
            int best = B.max_ctas_per_sm;
            if (any_render && B.autotune && B.max_ctas_per_sm > 1) {
                float best_ms = 3.4e38f;
                cudaEvent_t e0, e1;
                cudaEventCreate(&e0);
                cudaEventCreate(&e1);
                for (int c = B.max_ctas_per_sm; c >= std::max(1, B.max_ctas_per_sm - 1); --c) {
                    cudaEventRecord(e0, st);
                    enqueue_step(B, n_frames, true, c, st);
                    cudaEventRecord(e1, st);
                    cudaEventSynchronize(e1);
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (ms < best_ms) {
                        best_ms = ms;
                        best = c;
                    }
                }
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
            }
            shape.ctas_per_sm = best;
            cudaEventRecord(B.done[pb], st);
            B.pending[pb] = true;
            // one graph per staging buffer: copy of the argument blocks from
            // it, counter reset, the persistent launch
            for (int i = 0; i < 2; ++i) {
                cudaStream_t cs;
                if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return VSG_ERR_CUDA;
                cudaGraph_t g = nullptr;
                cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
                cudaMemcpyAsync(B.d_step, B.h_step[i], bytes, cudaMemcpyHostToDevice, cs);
                enqueue_step(B, n_frames, false, best, cs);
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
