// vsg_noalloc.cu -- frame integration that allocates no device memory.
//
// vsg_integrate keeps two per-pixel work buffers inside the scene (each
// pixel's world point with its camera distance, and its packed colour) and
// grows them with cudaMalloc the first time it sees a larger image.  Some
// callers cannot let that happen:
//   - plug-in hosts whose own allocator owns all device memory and forbids
//     the libraries it loads from calling cudaMalloc;
//   - real-time loops that must never stall on cudaMalloc / cudaFree, which
//     can synchronise the whole device;
//   - hosts that hand the library a fixed GPU memory budget at start-up and
//     forbid any allocation afterwards.
// vsg_integrate_noalloc runs the same integration with those work buffers
// taken from one fixed array of device memory compiled into this file, so
// the caller passes only its inputs (and the scene, created beforehand).
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/vsg.h"
#include "vsg_device.cuh"
#include "vsg_internal.h"

namespace {

// Largest frame the fixed work array serves: 1,048,576 pixels (1280x800
// fits; 1280x720 and 640x480 do).  Per pixel 16 bytes (float4 world point +
// camera distance) and 4 bytes (packed colour): 20 MiB, held by every GPU
// that loads the library until the process exits.
constexpr size_t kMaxPixels = size_t(1) << 20;
constexpr size_t kWorldBytes = kMaxPixels * sizeof(float4);
constexpr size_t kScratchBytes = kWorldBytes + kMaxPixels * sizeof(uint32_t);

static __device__ __align__(256) unsigned char g_pixel_scratch[kScratchBytes];

// The array's device address.  In host code the name g_pixel_scratch is only
// a host-side stand-in for the symbol, never a device address, so kernels
// must be given the address that cudaGetSymbolAddress returns with the
// device current.  That address belongs to the device's current context: it
// is looked up on the first call on each device and cached together with the
// context's unique id (cuCtxGetId), and looked up again whenever the id
// differs -- after cudaDeviceReset, or when the caller made another driver
// context current -- because the module, and with it the array, may then sit
// at another address.  Where the driver offers no context id, nothing is
// cached and every call looks the address up.
constexpr int kMaxDevices = 64;
struct ScratchSlot {
    unsigned long long ctx_id = 0;
    void* addr = nullptr;
};
std::mutex g_mutex;
ScratchSlot g_slot[kMaxDevices];

using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// The current context's unique id; false without a current context or
// without cuCtxGetId in the driver.
bool current_context_id(unsigned long long* id) {
    static CtxGetIdFn fn = []() -> CtxGetIdFn {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<CtxGetIdFn>(f);
    }();
    return fn && fn(nullptr, id) == CUDA_SUCCESS;
}

int scratch_for_device(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kMaxDevices) return VSG_ERR_TOO_LARGE;
    std::lock_guard<std::mutex> lock(g_mutex);
    unsigned long long id = 0;
    bool have_id = current_context_id(&id);
    if (have_id && g_slot[dev].addr && g_slot[dev].ctx_id == id) {
        *out = static_cast<unsigned char*>(g_slot[dev].addr);
        return VSG_OK;
    }
    void* p = nullptr;
    // runs with `dev` current: the caller's current device
    if (cudaGetSymbolAddress(&p, g_pixel_scratch) != cudaSuccess || p == nullptr) return VSG_ERR_CUDA;
    if (!have_id) have_id = current_context_id(&id);  // the lookup made the primary context current
    g_slot[dev].ctx_id = have_id ? id : 0;
    g_slot[dev].addr = have_id ? p : nullptr;
    *out = static_cast<unsigned char*>(p);
    return VSG_OK;
}

}  // namespace

extern "C" int vsg_integrate_noalloc(vsg_scene* s, const float* pointmap, const uint8_t* rgb, const float* normals,
                                     int w, int h, float truncation, const float pose[16], float fx, float fy,
                                     float cx, float cy, vsg_stream_t stream) {
    if (!s) return VSG_ERR_NOT_ALLOCATED;
    if (!pointmap || !rgb || !normals || !pose) return VSG_ERR_INVALID_ARG;
    if (w <= 0 || h <= 0) return VSG_ERR_INVALID_ARG;
    if ((size_t)w * (size_t)h > kMaxPixels) return VSG_ERR_TOO_LARGE;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return VSG_ERR_CUDA;
    if (dev != s->impl.device) return VSG_ERR_INVALID_ARG;  // the scene lives on another GPU
    unsigned char* base = nullptr;
    const int rc = scratch_for_device(dev, &base);
    if (rc != VSG_OK) return rc;
    // Nothing in the array needs clearing: the allocation kernel writes both
    // entries of every pixel of this frame before the integration kernel
    // reads any of them, and entries beyond w*h are never read.
    float4* pix_world = reinterpret_cast<float4*>(base);
    uint32_t* pix_rgb = reinterpret_cast<uint32_t*>(base + kWorldBytes);
    return vsg::scene_integrate_with_pixels(&s->impl, pointmap, rgb, w, h, truncation, pose, fx, fy, cx, cy,
                                            pix_world, pix_rgb, (cudaStream_t)stream);
}
