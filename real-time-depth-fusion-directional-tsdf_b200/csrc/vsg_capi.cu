// vsg_capi.cu -- the C ABI of include/vsg.h over the scene / renderer objects.
//
// Error behaviour: where the reference prints and returns void (null
// pointers VoxelScene.cpp:420-428, RayCastRender.cpp:128-136; launch
// errors VoxelScene.cu:1495-1502) these functions return a status code and
// print nothing.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <filesystem>
#include <new>
#include <vector>

#include "../../include/vsg.h"
#include "vsg_device.cuh"
#include "vsg_internal.h"

using vsg::Renderer;
using vsg::Scene;

namespace vsg {

void timing_begin(Scene* sc, int slot, cudaStream_t st) {
    Timing& t = sc->timing;
    if (!t.enabled) return;
    if (!t.created) {
        for (int i = 0; i < kNumSlots; ++i)
            for (int j = 0; j < Timing::kRing; ++j) {
                cudaEventCreate(&t.ev[i][j][0]);
                cudaEventCreate(&t.ev[i][j][1]);
            }
        t.created = true;
    }
    if (t.pending[slot] == Timing::kRing) {
        // ring full: fold the oldest pair in (synchronises on it)
        const int j = (t.head[slot] - t.pending[slot] + Timing::kRing) % Timing::kRing;
        float ms = 0.0f;
        cudaEventSynchronize(t.ev[slot][j][1]);
        cudaEventElapsedTime(&ms, t.ev[slot][j][0], t.ev[slot][j][1]);
        t.ms[slot] += ms;
        t.count[slot]++;
        t.pending[slot]--;
    }
    cudaEventRecord(t.ev[slot][t.head[slot]][0], st);
}

void timing_end(Scene* sc, int slot, cudaStream_t st) {
    Timing& t = sc->timing;
    if (!t.enabled) return;
    cudaEventRecord(t.ev[slot][t.head[slot]][1], st);
    t.head[slot] = (t.head[slot] + 1) % Timing::kRing;
    t.pending[slot]++;
}

static void timing_drain(Scene* sc) {
    Timing& t = sc->timing;
    if (!t.created) return;
    for (int s = 0; s < kNumSlots; ++s) {
        while (t.pending[s] > 0) {
            const int j = (t.head[s] - t.pending[s] + Timing::kRing) % Timing::kRing;
            float ms = 0.0f;
            cudaEventSynchronize(t.ev[s][j][1]);
            cudaEventElapsedTime(&ms, t.ev[s][j][0], t.ev[s][j][1]);
            t.ms[s] += ms;
            t.count[s]++;
            t.pending[s]--;
        }
    }
}

static void timing_destroy(Scene* sc) {
    Timing& t = sc->timing;
    if (!t.created) return;
    for (int i = 0; i < kNumSlots; ++i)
        for (int j = 0; j < Timing::kRing; ++j) {
            cudaEventDestroy(t.ev[i][j][0]);
            cudaEventDestroy(t.ev[i][j][1]);
        }
    t.created = false;
}

}  // namespace vsg

extern "C" {

const char* vsg_version(void) { return "vsg-b200 0.1 (sm_100a)"; }

int vsg_params_default(vsg_params* p) {
    if (!p) return VSG_ERR_INVALID_ARG;
    p->voxel_size = 0.004f;
    p->truncation = 0.02f;
    p->truncation_scale = 0.01f;
    p->hash_num_slots = 200000u;
    p->num_sdf_blocks = 200000u;
    p->max_chain_nodes = 0u;
    p->occupancy_log2 = 0u;
    return VSG_OK;
}

int vsg_scene_create(const vsg_params* p, vsg_scene** out) {
    if (!p || !out) return VSG_ERR_INVALID_ARG;
    *out = nullptr;
    // GlobalParamsConfig::validateParameters analogue (globalParamasConfig.cpp:404-417)
    if (!(p->voxel_size > 0.0f) || p->hash_num_slots == 0u || p->num_sdf_blocks == 0u) return VSG_ERR_INVALID_ARG;
    if (p->num_sdf_blocks > (1u << 26) || p->hash_num_slots > (1u << 28)) return VSG_ERR_TOO_LARGE;
    // (pools above 2^22 - 3 blocks resolve every block through the hash)
    if (p->occupancy_log2 > 9u || (p->occupancy_log2 != 0u && p->occupancy_log2 < 5u)) return VSG_ERR_TOO_LARGE;
    vsg_scene* h = new (std::nothrow) vsg_scene();
    if (!h) return VSG_ERR_OUT_OF_MEMORY;
    Scene& sc = h->impl;
    sc.params = *p;
    if (sc.params.max_chain_nodes == 0u) sc.params.max_chain_nodes = 2u * p->hash_num_slots;
    sc.bidx_log2 = p->occupancy_log2 ? (int)p->occupancy_log2 : 7;
    if (cudaGetDevice(&sc.device) != cudaSuccess) {
        delete h;
        return VSG_ERR_CUDA;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, sc.device);
    sc.sm_count = sms > 0 ? sms : 148;
    int rc = vsg::scene_alloc_device(&sc);
    if (rc != VSG_OK) {
        vsg::scene_free_device(&sc);
        delete h;
        return rc;
    }
    rc = vsg::scene_reset_device(&sc, 0);
    if (rc == VSG_OK && cudaStreamSynchronize(0) != cudaSuccess) rc = VSG_ERR_CUDA;
    if (rc != VSG_OK) {
        vsg::scene_free_device(&sc);
        delete h;
        return rc;
    }
    *out = h;
    return VSG_OK;
}

int vsg_scene_destroy(vsg_scene* s) {
    if (!s) return VSG_ERR_INVALID_ARG;
    cudaDeviceSynchronize();
    vsg::timing_destroy(&s->impl);
    vsg::stream_stage_free(&s->impl);
    vsg::scene_free_device(&s->impl);
    delete s;
    return VSG_OK;
}

// True when the calling thread's current device is `device`: a scene's hash,
// pool and counters, and a renderer's outputs, live on the device current at
// their creation, and kernels launched on another device would dereference
// that device's pointers.
static bool on_device(int device) {
    int dev = -1;
    return cudaGetDevice(&dev) == cudaSuccess && dev == device;
}

int vsg_scene_reset(vsg_scene* s, vsg_stream_t stream) {
    if (!s) return VSG_ERR_INVALID_ARG;
    if (!on_device(s->impl.device)) return VSG_ERR_INVALID_ARG;
    return vsg::scene_reset_device(&s->impl, (cudaStream_t)stream);
}

int vsg_scene_params(const vsg_scene* s, vsg_params* out) {
    if (!s || !out) return VSG_ERR_INVALID_ARG;
    *out = s->impl.params;
    return VSG_OK;
}

int vsg_integrate(vsg_scene* s, const float* pointmap, const uint8_t* rgb, const float* normals, int w, int h,
                  float truncation, const float pose[16], float fx, float fy, float cx, float cy,
                  vsg_stream_t stream) {
    if (!s) return VSG_ERR_NOT_ALLOCATED;
    if (!pointmap || !rgb || !normals || !pose) return VSG_ERR_INVALID_ARG;
    if (w <= 0 || h <= 0 || (long long)w * h > (1ll << 30)) return VSG_ERR_INVALID_ARG;
    if (!on_device(s->impl.device)) return VSG_ERR_INVALID_ARG;
    return vsg::scene_integrate(&s->impl, pointmap, rgb, normals, w, h, truncation, pose, fx, fy, cx, cy,
                                (cudaStream_t)stream);
}

int vsg_scene_set_alloc_method(vsg_scene* s, int method) {
    if (!s) return VSG_ERR_NOT_ALLOCATED;
    if (method != 1 && method != 2) return VSG_ERR_INVALID_ARG;
    s->impl.dev.alloc_method = method;
    return VSG_OK;
}

int vsg_scene_stats(vsg_scene* s, vsg_stats* out) {
    if (!s || !out) return VSG_ERR_INVALID_ARG;
    // the synchronisation below waits for the current device only
    if (!on_device(s->impl.device)) return VSG_ERR_INVALID_ARG;
    if (cudaDeviceSynchronize() != cudaSuccess) return VSG_ERR_CUDA;
    vsg::SceneCounters c;
    vsg::FrameCounters f;
    if (cudaMemcpy(&c, s->impl.dev.ctr, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess) return VSG_ERR_CUDA;
    if (cudaMemcpy(&f, s->impl.dev.frame, sizeof(f), cudaMemcpyDeviceToHost) != cudaSuccess) return VSG_ERR_CUDA;
    memset(out, 0, sizeof(*out));
    const int B = s->impl.dev.num_blocks;
    out->free_blocks = (uint32_t)std::max(c.free_count, 0);
    out->allocated_blocks = (uint32_t)(B - std::max(c.free_count, 0));
    out->high_water = c.high_water;
    out->chain_nodes_used = (uint32_t)std::min(c.nodes_used, s->impl.dev.max_nodes);
    out->integrated_frames = s->impl.integrated_frames;
    out->frame_valid_pixels = f.n_valid_px;
    out->frame_new_blocks = f.n_new;
    out->frame_visible_blocks = f.n_visible;
    out->frame_updated_blocks = f.n_upd_blocks;
    out->frame_updated_voxels = f.n_upd_voxels;
    out->render_hits = f.hits;
    out->render_misses = f.misses;
    out->render_samples_full = f.samples_full;
    out->render_samples_skipped = f.samples_skipped;
    out->render_jumps = f.jumps;
    out->render_singles = f.singles;
    out->render_blocks_read = f.blocks_read;
    out->render_lane_iters = f.lane_iters;
    out->render_warp_iters = f.warp_iters;
    out->flags = c.flags;
    out->fast_division = s->impl.dev.div_fast ? 1u : 0u;
    {
        float tab[257];
        if (cudaMemcpy(tab, s->impl.dev.avg_recip, sizeof(tab), cudaMemcpyDeviceToHost) != cudaSuccess)
            return VSG_ERR_CUDA;
        for (int d = 1; d <= 256; ++d) out->fast_avg_divisors += tab[d] != 0.0f ? 1u : 0u;
    }
    out->pixel_buffer_capacity = (uint32_t)std::min<size_t>(s->impl.pix_capacity, UINT32_MAX);
    return VSG_OK;
}

int vsg_scene_export(vsg_scene* s, int32_t* coords, uint8_t* voxels, uint32_t max_blocks, uint32_t* n_out) {
    return vsg::host_guard([&]() -> int {
        if (!s || !coords || !n_out) return VSG_ERR_INVALID_ARG;
        if (!on_device(s->impl.device)) return VSG_ERR_INVALID_ARG;
        if (cudaDeviceSynchronize() != cudaSuccess) return VSG_ERR_CUDA;
        vsg::SceneCounters c;
        if (cudaMemcpy(&c, s->impl.dev.ctr, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess) return VSG_ERR_CUDA;
        const uint32_t hw = c.high_water;
        std::vector<unsigned long long> keys(hw);
        if (hw && cudaMemcpy(keys.data(), s->impl.dev.block_key, hw * sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost) != cudaSuccess)
            return VSG_ERR_CUDA;
        std::vector<std::pair<std::array<int, 3>, uint32_t>> live;
        live.reserve(hw);
        for (uint32_t i = 0; i < hw; ++i) {
            if (keys[i] == vsg::kKeyEmpty || keys[i] == vsg::kKeyTomb) continue;
            int x, y, z;
            vsg::unpack_key(keys[i], x, y, z);
            live.push_back({{x, y, z}, i});
        }
        *n_out = (uint32_t)live.size();
        if (live.size() > max_blocks) return VSG_ERR_TOO_LARGE;
        std::sort(live.begin(), live.end());
        std::vector<vsg::Voxel> vox;
        if (voxels && hw) {
            vox.resize((size_t)hw * vsg::kVoxPerBlock);
            if (cudaMemcpy(vox.data(), s->impl.dev.voxels, vox.size() * sizeof(vsg::Voxel), cudaMemcpyDeviceToHost) !=
                cudaSuccess)
                return VSG_ERR_CUDA;
        }
        for (size_t i = 0; i < live.size(); ++i) {
            coords[3 * i + 0] = live[i].first[0];
            coords[3 * i + 1] = live[i].first[1];
            coords[3 * i + 2] = live[i].first[2];
            if (voxels)
                memcpy(voxels + i * vsg::kVoxPerBlock * 8, vox.data() + (size_t)live[i].second * vsg::kVoxPerBlock,
                       vsg::kVoxPerBlock * 8);
        }
        return VSG_OK;
    });
}

int vsg_renderer_create(int w, int h, vsg_renderer** out) {
    if (!out || w <= 0 || h <= 0 || (long long)w * h > (1ll << 30)) return VSG_ERR_INVALID_ARG;
    *out = nullptr;
    vsg_renderer* r = new (std::nothrow) vsg_renderer();
    if (!r) return VSG_ERR_OUT_OF_MEMORY;
    Renderer& R = r->impl;
    R.w = w;
    R.h = h;
    cudaGetDevice(&R.device);
    cudaDeviceGetAttribute(&R.sm_count, cudaDevAttrMultiProcessorCount, R.device);
    const size_t n = (size_t)w * h;
    // RayCastRender::initialize, RayCastRender.cpp:88-118
    const size_t nb = (size_t)((w + 7) / 8) * ((h + 3) / 4) + (size_t)((w + 63) / 64) * ((h + 31) / 32) + 1;
    if (cudaMalloc(&R.depth, n * sizeof(float)) != cudaSuccess || cudaMalloc(&R.position, n * sizeof(float4)) != cudaSuccess ||
        cudaMalloc(&R.color, n * sizeof(float4)) != cudaSuccess || cudaMalloc(&R.normal, n * sizeof(float4)) != cudaSuccess ||
        cudaMalloc(&R.bounds, nb * sizeof(uint2)) != cudaSuccess ||
        cudaMalloc(&R.tile_order, (size_t)((w + 15) / 16) * ((h + 7) / 8) * sizeof(uint32_t)) != cudaSuccess) {
        cudaFree(R.tile_order);
        cudaFree(R.depth);
        cudaFree(R.position);
        cudaFree(R.color);
        cudaFree(R.normal);
        cudaFree(R.bounds);
        delete r;
        return VSG_ERR_OUT_OF_MEMORY;
    }
    *out = r;
    return VSG_OK;
}

int vsg_renderer_destroy(vsg_renderer* r) {
    if (!r) return VSG_ERR_INVALID_ARG;
    cudaDeviceSynchronize();
    cudaFree(r->impl.depth);
    cudaFree(r->impl.position);
    cudaFree(r->impl.color);
    cudaFree(r->impl.normal);
    cudaFree(r->impl.bounds);
    cudaFree(r->impl.tile_order);
    cudaFree(r->impl.bracket);
    cudaFree(r->impl.partials);
    cudaFree(r->impl.skipped);
    delete r;
    return VSG_OK;
}

int vsg_render(vsg_renderer* r, const vsg_scene* s, const float cam_pos[3], const float* pose_dev, float fx,
               float fy, float cx, float cy, float min_depth, float max_depth, vsg_stream_t stream) {
    if (!r) return VSG_ERR_NOT_ALLOCATED;
    if (!s || !cam_pos || !pose_dev) return VSG_ERR_INVALID_ARG;
    if (!on_device(s->impl.device) || !on_device(r->impl.device)) return VSG_ERR_INVALID_ARG;
    return vsg::render_launch(&r->impl, const_cast<Scene*>(&s->impl), cam_pos, pose_dev, nullptr, fx, fy, cx, cy,
                              min_depth, max_depth, (cudaStream_t)stream);
}

int vsg_render_hostpose(vsg_renderer* r, const vsg_scene* s, const float cam_pos[3], const float pose[16], float fx,
                        float fy, float cx, float cy, float min_depth, float max_depth, vsg_stream_t stream) {
    if (!r) return VSG_ERR_NOT_ALLOCATED;
    if (!s || !cam_pos || !pose) return VSG_ERR_INVALID_ARG;
    if (!on_device(s->impl.device) || !on_device(r->impl.device)) return VSG_ERR_INVALID_ARG;
    return vsg::render_launch(&r->impl, const_cast<Scene*>(&s->impl), cam_pos, nullptr, pose, fx, fy, cx, cy,
                              min_depth, max_depth, (cudaStream_t)stream);
}

int vsg_renderer_set_step(vsg_renderer* r, float step) {
    if (!r) return VSG_ERR_NOT_ALLOCATED;
    if (!(step >= 0.0f) || !std::isfinite(step)) return VSG_ERR_INVALID_ARG;
    r->impl.step = step;
    return VSG_OK;
}

int vsg_renderer_outputs(const vsg_renderer* r, float** depth, float** position, float** color, float** normal) {
    if (!r) return VSG_ERR_INVALID_ARG;
    if (depth) *depth = r->impl.depth;
    if (position) *position = (float*)r->impl.position;
    if (color) *color = (float*)r->impl.color;
    if (normal) *normal = (float*)r->impl.normal;
    return VSG_OK;
}

int vsg_renderer_download(const vsg_renderer* r, float* depth, float* position, float* color, float* normal) {
    if (!r) return VSG_ERR_INVALID_ARG;
    if (!on_device(r->impl.device)) return VSG_ERR_INVALID_ARG;
    const size_t n = (size_t)r->impl.w * r->impl.h;
    if (cudaDeviceSynchronize() != cudaSuccess) return VSG_ERR_CUDA;
    if (depth && cudaMemcpy(depth, r->impl.depth, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return VSG_ERR_CUDA;
    if (position && cudaMemcpy(position, r->impl.position, n * 16, cudaMemcpyDeviceToHost) != cudaSuccess)
        return VSG_ERR_CUDA;
    if (color && cudaMemcpy(color, r->impl.color, n * 16, cudaMemcpyDeviceToHost) != cudaSuccess) return VSG_ERR_CUDA;
    if (normal && cudaMemcpy(normal, r->impl.normal, n * 16, cudaMemcpyDeviceToHost) != cudaSuccess)
        return VSG_ERR_CUDA;
    return VSG_OK;
}

int vsg_renderer_save_ply(const vsg_renderer* r, const char* path, int64_t* n_points) {
    return vsg::host_guard([&]() -> int {
        if (!r || !path) return VSG_ERR_INVALID_ARG;
        if (n_points) *n_points = 0;
        const size_t n = (size_t)r->impl.w * r->impl.h;
        std::vector<float> D(n);
        std::vector<float4> P(n), C(n);
        int rc = vsg_renderer_download(r, D.data(), reinterpret_cast<float*>(P.data()),
                                       reinterpret_cast<float*>(C.data()), nullptr);
        if (rc != VSG_OK) return rc;
        auto valid = [&](size_t i) {
            return std::isfinite(D[i]) && D[i] > 0.0f && std::fabs(D[i]) < 1e9f && std::isfinite(P[i].x) &&
                   std::isfinite(P[i].y) && std::isfinite(P[i].z);
        };
        int64_t count = 0;
        for (size_t i = 0; i < n; ++i) count += valid(i) ? 1 : 0;
        if (count == 0) return VSG_ERR_INVALID_ARG;
        std::error_code ec;
        const std::filesystem::path out(path);
        if (out.has_parent_path()) std::filesystem::create_directories(out.parent_path(), ec);
        FILE* f = std::fopen(path, "w");
        if (!f) return VSG_ERR_INVALID_ARG;
        std::fprintf(f,
                     "ply\nformat ascii 1.0\ncomment Generated by RayCastRender\nelement vertex %lld\n"
                     "property float x\nproperty float y\nproperty float z\n"
                     "property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n",
                     (long long)count);
        auto channel = [](float c) -> int {
            if (!std::isfinite(c)) return 255;
            c = c < 0.0f ? 0.0f : (c > 1.0f ? 1.0f : c);
            return static_cast<int>(c * 255.0f + 0.5f);
        };
        for (size_t i = 0; i < n; ++i) {
            if (!valid(i)) continue;
            std::fprintf(f, "%g %g %g %d %d %d\n", P[i].x, P[i].y, P[i].z, channel(C[i].x), channel(C[i].y),
                         channel(C[i].z));
        }
        if (std::fclose(f) != 0) return VSG_ERR_INVALID_ARG;
        if (n_points) *n_points = count;
        return VSG_OK;
    });
}

int vsg_timing_enable(vsg_scene* s, int enable) {
    if (!s) return VSG_ERR_INVALID_ARG;
    s->impl.timing.enabled = enable != 0;
    return VSG_OK;
}

int vsg_scene_march_stats(vsg_scene* s, int enable) {
    if (!s) return VSG_ERR_INVALID_ARG;
    s->impl.march_stats = enable != 0;
    return VSG_OK;
}

int vsg_timing_read(vsg_scene* s, double* ms, uint32_t* counts, int n_slots) {
    if (!s || !ms || !counts || n_slots <= 0) return VSG_ERR_INVALID_ARG;
    vsg::timing_drain(&s->impl);
    for (int i = 0; i < n_slots && i < vsg::kNumSlots; ++i) {
        ms[i] = s->impl.timing.ms[i];
        counts[i] = s->impl.timing.count[i];
    }
    return VSG_OK;
}

int vsg_timing_reset(vsg_scene* s) {
    if (!s) return VSG_ERR_INVALID_ARG;
    vsg::timing_drain(&s->impl);
    for (int i = 0; i < vsg::kNumSlots; ++i) {
        s->impl.timing.ms[i] = 0.0;
        s->impl.timing.count[i] = 0;
    }
    return VSG_OK;
}

}  // extern "C"
