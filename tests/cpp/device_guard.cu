// A scene or renderer used with another device current must be refused
// before any launch.  One GPU cannot make a second device current, so the
// harness records another device ordinal in the handles (the field the entry
// points compare against the current device) and checks that
// vsg_integrate, vsg_scene_reset, vsg_render, vsg_render_hostpose,
// vsg_scene_stats, vsg_scene_export, vsg_scene_lookup_blocks,
// vsg_renderer_record, vsg_renderer_download and vsg_batch_create return
// VSG_ERR_INVALID_ARG and leave the scene, the renderer and the outputs
// untouched; with the true ordinal restored the same calls succeed.  Prints
// "device_guard ok" on success.
#include <cstdio>
#include <cstring>

#include <cuda_runtime.h>

#include "vsg.h"
#include "vsg_internal.h"

#define CHECK(cond)                                                        \
    do {                                                                   \
        if (!(cond)) {                                                     \
            std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond); \
            return 1;                                                      \
        }                                                                  \
    } while (0)

int main() {
    const int W = 64, H = 48;
    vsg_params p;
    CHECK(vsg_params_default(&p) == VSG_OK);
    p.hash_num_slots = 1021;
    p.num_sdf_blocks = 4000;
    vsg_scene* s = nullptr;
    vsg_renderer* r = nullptr;
    CHECK(vsg_scene_create(&p, &s) == VSG_OK);
    CHECK(vsg_renderer_create(W, H, &r) == VSG_OK);
    float* pm = nullptr;
    uint8_t* rgb = nullptr;
    float* nm = nullptr;
    float* pose_dev = nullptr;
    CHECK(cudaMalloc(&pm, W * H * 12) == cudaSuccess);
    CHECK(cudaMalloc(&rgb, W * H * 3) == cudaSuccess);
    CHECK(cudaMalloc(&nm, W * H * 12) == cudaSuccess);
    CHECK(cudaMalloc(&pose_dev, 64) == cudaSuccess);
    // a fronto-parallel wall 1 m in front of the camera
    float host_pm[W * H * 3];
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            host_pm[3 * (y * W + x) + 0] = (x - 31.5f) / 50.0f;
            host_pm[3 * (y * W + x) + 1] = (y - 23.5f) / 50.0f;
            host_pm[3 * (y * W + x) + 2] = 1.0f;
        }
    CHECK(cudaMemcpy(pm, host_pm, sizeof(host_pm), cudaMemcpyHostToDevice) == cudaSuccess);
    CHECK(cudaMemset(rgb, 128, W * H * 3) == cudaSuccess);
    CHECK(cudaMemset(nm, 0, W * H * 12) == cudaSuccess);
    float pose[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    CHECK(cudaMemcpy(pose_dev, pose, 64, cudaMemcpyHostToDevice) == cudaSuccess);
    const float cam[3] = {0, 0, 0};

    int dev = -1;
    CHECK(cudaGetDevice(&dev) == cudaSuccess);
    CHECK(s->impl.device == dev && r->impl.device == dev);

    vsg_stats st;
    int32_t coords[3] = {0, 0, 0};
    int32_t ptrs[1] = {-7};
    uint32_t n_out = 123u;
    static float depth_h[W * H];
    vsg_batch* b = nullptr;

    s->impl.device = dev + 1;  // the scene now claims another GPU
    CHECK(vsg_integrate(s, pm, rgb, nm, W, H, 0.02f, pose, 50, 50, 31.5f, 23.5f, 0) == VSG_ERR_INVALID_ARG);
    CHECK(vsg_scene_reset(s, 0) == VSG_ERR_INVALID_ARG);
    CHECK(vsg_render(r, s, cam, pose_dev, 50, 50, 31.5f, 23.5f, 0.2f, 3.0f, 0) == VSG_ERR_INVALID_ARG);
    CHECK(vsg_render_hostpose(r, s, cam, pose, 50, 50, 31.5f, 23.5f, 0.2f, 3.0f, 0) == VSG_ERR_INVALID_ARG);
    CHECK(vsg_scene_stats(s, &st) == VSG_ERR_INVALID_ARG);
    CHECK(vsg_scene_export(s, coords, nullptr, 1u, &n_out) == VSG_ERR_INVALID_ARG && n_out == 123u);
    CHECK(vsg_scene_lookup_blocks(s, coords, 1u, ptrs) == VSG_ERR_INVALID_ARG && ptrs[0] == -7);
    CHECK(vsg_batch_create(&s, &r, 1, &b) == VSG_ERR_INVALID_ARG && b == nullptr);
    s->impl.device = dev;
    r->impl.device = dev + 1;  // the renderer now claims another GPU
    CHECK(vsg_render(r, s, cam, pose_dev, 50, 50, 31.5f, 23.5f, 0.2f, 3.0f, 0) == VSG_ERR_INVALID_ARG);
    CHECK(vsg_render_hostpose(r, s, cam, pose, 50, 50, 31.5f, 23.5f, 0.2f, 3.0f, 0) == VSG_ERR_INVALID_ARG);
    CHECK(vsg_renderer_record(r, 1) == VSG_ERR_INVALID_ARG && r->impl.bracket == nullptr);
    CHECK(vsg_renderer_download(r, depth_h, nullptr, nullptr, nullptr) == VSG_ERR_INVALID_ARG);
    CHECK(vsg_batch_create(&s, &r, 1, &b) == VSG_ERR_INVALID_ARG && b == nullptr);
    r->impl.device = dev;

    CHECK(vsg_scene_stats(s, &st) == VSG_OK);
    CHECK(st.integrated_frames == 0 && st.allocated_blocks == 0);
    // with the true ordinals the refused calls run
    CHECK(vsg_batch_create(&s, &r, 1, &b) == VSG_OK && b != nullptr);
    CHECK(vsg_batch_destroy(b) == VSG_OK);
    CHECK(vsg_renderer_record(r, 1) == VSG_OK && r->impl.bracket != nullptr);
    CHECK(vsg_renderer_record(r, 0) == VSG_OK);

    // the true ordinal: the same calls run
    CHECK(vsg_integrate(s, pm, rgb, nm, W, H, 0.02f, pose, 50, 50, 31.5f, 23.5f, 0) == VSG_OK);
    CHECK(vsg_render(r, s, cam, pose_dev, 50, 50, 31.5f, 23.5f, 0.2f, 3.0f, 0) == VSG_OK);
    CHECK(vsg_render_hostpose(r, s, cam, pose, 50, 50, 31.5f, 23.5f, 0.2f, 3.0f, 0) == VSG_OK);
    CHECK(vsg_scene_stats(s, &st) == VSG_OK);
    CHECK(st.integrated_frames == 1 && st.allocated_blocks > 0 && st.render_hits > 0);
    CHECK(vsg_renderer_download(r, depth_h, nullptr, nullptr, nullptr) == VSG_OK);
    CHECK(vsg_scene_export(s, coords, nullptr, 0u, &n_out) == VSG_ERR_TOO_LARGE && n_out > 0u);
    CHECK(vsg_scene_lookup_blocks(s, coords, 1u, ptrs) == VSG_OK);
    CHECK(vsg_scene_reset(s, 0) == VSG_OK);
    CHECK(cudaDeviceSynchronize() == cudaSuccess);

    cudaFree(pm);
    cudaFree(rgb);
    cudaFree(nm);
    cudaFree(pose_dev);
    vsg_renderer_destroy(r);
    vsg_scene_destroy(s);
    std::printf("device_guard ok\n");
    return 0;
}
