// vsg_device.cuh -- data layout in HBM and device helpers shared by the
// fusion kernels.
//
// Layout (one scene):
//   buckets     Entry[S * 8]      16-B entries {u64 key, i32 ptr, i32 aux};
//                                 a bucket is one 128-B line
//   bucket_next i32[S]            head of the bucket's overflow chain (-1)
//   nodes       Node[M]           overflow entries {u64 key, i32 ptr, i32 next}
//   voxels      Voxel[B * 512]    8-B voxels {f32 sdf, u32 r|g<<8|b<<16|w<<24},
//                                 block-major, x fastest (x + 8y + 64z)
//   block_key   u64[B]            pool block -> packed coordinate (EMPTY = free)
//   block_slot  i32[B]            pool block -> entry index (>= S*8: chain node)
//   block_fresh u8[B]             1 until the block's first integration pass
//   heap        u32[B]            free-list stack of pool indices
//   occ_raw     u32[cells/32]     toroidal bit per allocated block
//   occ_dil     u32[cells/32]     same, dilated by one block in every direction
//
// Packed block key: 21-bit two's complement per axis, x in bits 42..62,
// y in 21..41, z in 0..20; ~0 = empty, ~0-1 = deleted (tombstone).
//
// Floating point on the path is compiled without FMA contraction
// (-fmad=false) so every expression rounds exactly like the reference's
// operation sequence; the comments give the reference file:line restated.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vsg {

constexpr int kBlock = 8;
constexpr int kVoxPerBlock = 512;
constexpr int kBucketSlots = 8;
constexpr unsigned long long kKeyEmpty = 0xFFFFFFFFFFFFFFFFull;
constexpr unsigned long long kKeyTomb = 0xFFFFFFFFFFFFFFFEull;
constexpr int kCoordLim = 1 << 20;
constexpr float kMinf = 1e10f;

struct __align__(16) Entry {
    unsigned long long key;
    int ptr;
    int aux;
};

struct __align__(16) Node {
    unsigned long long key;
    int ptr;
    int next;
};

struct __align__(8) Voxel {
    float sdf;
    uint32_t rgbw;
};

// persistent per-scene counters (device)
struct SceneCounters {
    int free_count;          // heap entries [0, free_count) are free
    uint32_t high_water;     // max pool index handed out + 1
    int nodes_used;          // overflow nodes consumed
    uint32_t flags;          // VSG_FLAG_* (sticky)
    uint32_t alloc_fail;     // blocks not allocated (pool or chain exhausted)
    uint32_t coord_drops;    // blocks outside the packable coordinate range
    uint32_t pad[2];
};

// per-frame counters (device), cleared before each frame
struct FrameCounters {
    uint32_t zmin_ord;       // ordered-int min camera z over pixels p != 0
    uint32_t zmax_ord;
    uint32_t nonfinite;      // a valid pixel holds inf/nan: disables culling
    uint32_t n_valid_px;     // pixels with p != 0
    uint32_t n_new;          // blocks allocated this frame
    uint32_t n_visible;      // blocks passed to integration
    uint32_t n_upd_blocks;   // blocks with >= 1 updated voxel
    uint32_t n_upd_voxels;   // voxels updated
    uint32_t chunk;          // integration work queue
    uint32_t hits;           // render counters
    uint32_t misses;
    uint32_t pad[5];
};

struct SceneDev {
    Entry* buckets;
    int* bucket_next;
    Node* nodes;
    Voxel* voxels;
    unsigned long long* block_key;
    int* block_slot;
    uint8_t* block_fresh;
    uint32_t* heap;
    uint32_t* occ_raw;
    uint32_t* occ_dil;
    uint32_t* visible;
    SceneCounters* ctr;
    FrameCounters* frame;
    uint32_t num_buckets;
    int num_blocks;
    int max_nodes;
    int occ_log2;
    float voxel;
};

struct Pose {
    float T[16];  // row-major camera->world
};

// ------------------------------------------------------------ key helpers

__host__ __device__ __forceinline__ bool coord_ok(int x, int y, int z) {
    return x >= -kCoordLim && x < kCoordLim && y >= -kCoordLim && y < kCoordLim && z >= -kCoordLim &&
           z < kCoordLim;
}

__host__ __device__ __forceinline__ unsigned long long pack_key(int x, int y, int z) {
    const unsigned long long m = 0x1FFFFFull;
    return (((unsigned long long)(unsigned)x & m) << 42) | (((unsigned long long)(unsigned)y & m) << 21) |
           ((unsigned long long)(unsigned)z & m);
}

__host__ __device__ __forceinline__ int sext21(unsigned long long v) {
    return (int)((int)((unsigned)(v & 0x1FFFFFull) << 11) >> 11);
}

__host__ __device__ __forceinline__ void unpack_key(unsigned long long k, int& x, int& y, int& z) {
    x = sext21(k >> 42);
    y = sext21(k >> 21);
    z = sext21(k);
}

// Bucket hash, VoxelScene.cu:61-66 (wrapping 32-bit products, unsigned mod).
__host__ __device__ __forceinline__ uint32_t bucket_of(int x, int y, int z, uint32_t nb) {
    uint32_t h = ((uint32_t)x * 73856093u) ^ ((uint32_t)y * 19349663u) ^ ((uint32_t)z * 83492791u);
    return h % nb;
}

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
    return *(const volatile unsigned long long*)p;
}

__device__ __forceinline__ int ld_volatile_i32(const int* p) { return *(const volatile int*)p; }

// ordered-int encoding of floats (monotone for non-NaN)
__device__ __forceinline__ uint32_t f2ord(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float ord2f(uint32_t u) {
    uint32_t b = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float f;
    __builtin_memcpy(&f, &b, 4);
    return f;
#endif
}

// --------------------------------------------------------- occupancy grid

__device__ __forceinline__ uint32_t occ_bit(int x, int y, int z, int lg) {
    const uint32_t m = (1u << lg) - 1u;
    return (((uint32_t)z & m) << (2 * lg)) | (((uint32_t)y & m) << lg) | ((uint32_t)x & m);
}

__device__ __forceinline__ bool occ_test(const uint32_t* occ, int x, int y, int z, int lg) {
    uint32_t b = occ_bit(x, y, z, lg);
    return (__ldg(occ + (b >> 5)) >> (b & 31)) & 1u;
}

// ------------------------------------------------------------ hash lookup

// Pool index of a block, or -1.  Buckets fill their first free slot, and a
// slot never returns to EMPTY once used, so an EMPTY slot ends the search
// (the overflow chain is only ever started by a full bucket).
__device__ __forceinline__ int lookup_block(const SceneDev& s, unsigned long long key, int x, int y, int z) {
    const uint32_t b = bucket_of(x, y, z, s.num_buckets);
    const Entry* bk = s.buckets + (size_t)b * kBucketSlots;
#pragma unroll
    for (int j = 0; j < kBucketSlots; ++j) {
        const uint4 e = __ldg(reinterpret_cast<const uint4*>(bk + j));
        const unsigned long long k = ((unsigned long long)e.y << 32) | e.x;
        if (k == key) return (int)e.z;
        if (k == kKeyEmpty) return -1;
    }
    int n = __ldg(s.bucket_next + b);
    for (int it = 0; n >= 0 && it < s.max_nodes; ++it) {
        const uint4 e = __ldg(reinterpret_cast<const uint4*>(s.nodes + n));
        const unsigned long long k = ((unsigned long long)e.y << 32) | e.x;
        if (k == key) return (int)e.z;
        n = (int)e.w;
    }
    return -1;
}

__device__ __forceinline__ uint32_t pack_rgbw(uint32_t r, uint32_t g, uint32_t b, uint32_t w) {
    return r | (g << 8) | (b << 16) | (w << 24);
}

}  // namespace vsg
