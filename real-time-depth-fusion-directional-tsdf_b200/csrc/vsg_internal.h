// vsg_internal.h -- host-side objects behind the opaque C handles.
#pragma once

#include <cuda_runtime.h>

#include "../../include/vsg.h"
#include "vsg_device.cuh"

#include <new>
#include <stdexcept>

namespace vsg {

// Host-side entry points run their body through this: an exception (host
// memory exhausted) becomes an error code instead of crossing the C ABI.
template <class F>
int host_guard(F&& f) noexcept {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return VSG_ERR_OUT_OF_MEMORY;
    } catch (const std::length_error&) {
        return VSG_ERR_OUT_OF_MEMORY;
    } catch (...) {
        return VSG_ERR_INVALID_ARG;
    }
}

enum TimingSlot {
    kSlotAlloc = 0,
    kSlotIntegrate = 1,
    kSlotRender = 2,
    kSlotSelect = 3,
    kSlotMarchingCubes = 4,
    kSlotExtractPoints = 5,
    kNumSlots = 8
};

struct Timing {
    bool enabled = false;
    static constexpr int kRing = 64;
    cudaEvent_t ev[kNumSlots][kRing][2] = {};
    int head[kNumSlots] = {};
    int pending[kNumSlots] = {};
    double ms[kNumSlots] = {};
    uint32_t count[kNumSlots] = {};
    bool created = false;
};

struct Scene {
    vsg_params params{};
    int bidx_log2 = 7;
    int sm_count = 148;
    int device = 0;
    SceneDev dev{};
    size_t pix_capacity = 0;  // pixels the per-frame buffers hold
    int integ_ctas_per_sm = 2;
    uint32_t integrated_frames = 0;
    Timing timing;
    bool march_stats = false;  // renders count skips, boundary samples and blocks read
    void* stream_stage = nullptr;  // staging buffers of vsg_stream_* (created on first use)
};

struct Renderer {
    int w = 0, h = 0;
    int device = 0;
    float* depth = nullptr;
    float4* position = nullptr;
    float4* color = nullptr;
    float4* normal = nullptr;
    uint2* bounds = nullptr;  // march distance bounds per pixel tile (k_tile_bounds)
    uint32_t* tile_order = nullptr;  // ray-cast CTA tiles, longest march range first (k_tile_order)
    int sm_count = 148;
    // adjoint support (vsg_renderer_record): march brackets, per-CTA pose
    // gradient partials, skipped-pixel counter
    bool record = false;
    float2* bracket = nullptr;
    double* partials = nullptr;
    unsigned int* skipped = nullptr;
    float step = 0.0f;  // march step in metres; 0 = the reference's half voxel
};

int scene_alloc_device(Scene* sc);
void scene_free_device(Scene* sc);
int scene_reset_device(Scene* sc, cudaStream_t st);
int scene_integrate(Scene* sc, const float* pm, const uint8_t* rgb, const float* nm, int W, int H, float trunc,
                    const float* pose, float fx, float fy, float cx, float cy, cudaStream_t st);
int ensure_pixel_buffers(Scene* sc, size_t npx);
int scene_integrate_with_pixels(Scene* sc, const float* pm, const uint8_t* rgb, int W, int H, float trunc,
                                const float* pose, float fx, float fy, float cx, float cy, float4* pix_world,
                                uint32_t* pix_rgb, cudaStream_t st);
int render_launch(Renderer* r, Scene* sc, const float cam[3], const float* pose_dev, const float* pose_host,
                  float fx, float fy, float cx, float cy, float min_depth, float max_depth, cudaStream_t st);

int verify_fixed_division(float v, bool* ok);

void stream_stage_free(Scene* sc);

void timing_begin(Scene* sc, int slot, cudaStream_t st);
void timing_end(Scene* sc, int slot, cudaStream_t st);

}  // namespace vsg

struct vsg_scene {
    vsg::Scene impl;
};
struct vsg_renderer {
    vsg::Renderer impl;
};
