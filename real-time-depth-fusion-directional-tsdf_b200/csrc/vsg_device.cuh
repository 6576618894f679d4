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
//   block_wmask u64[B]            bit (sz*4+sy)*4+sx: sub-cube (2x2x2 voxels)
//                                 holds a voxel with weight > 0
//   heap        u32[B]            free-list stack of pool indices
//   bindex      u64[2^(3k)]       dense toroidal block index: cell (x,y,z) mod 2^k
//                                 holds ptr (22 bits) | high coordinate bits
//                                 (tag) << 22 of the one block mapped there;
//                                 ~0 = none, ~0-1 = several (use the hash)
//   dwm         u64[2^(3k)]       per toroidal block position: sub-cubes that
//                                 have a weighted sub-cube within one sub-cube
//                                 (3x3x3, across block faces); ray-march skip
//   sup         u32[2^(3(k-3))/32] per toroidal super-cell (8^3 block
//                                 positions): some dwm word in it is non-zero
//   visible     u32[B]            pool indices the current frame integrates
//   pix_world   float4[W*H]       per pixel of the current frame: world point
//                                 T*p and its camera distance (-1: invalid)
//   pix_rgb     u32[W*H]          per pixel colour, packed
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
    uint32_t chunk;          // selection / integration work queues
    uint32_t work;
    uint32_t hits;           // render counters
    uint32_t misses;
    uint32_t samples_full;   // march samples evaluated with trilinear taps
    uint32_t samples_skipped;  // march samples skipped as provably invalid
    uint32_t jumps;          // O(1) jumps over runs of skipped samples
    uint32_t singles;        // samples evaluated at a cell boundary (no jump)
    uint32_t blocks_read;    // distinct blocks the last render read (instrumented runs)
    uint32_t lane_iters;     // march loop iterations summed over rays (x1/32 per warp)
    uint32_t warp_iters;     // per-warp maximum iterations summed over warps
    uint32_t n_parent;       // normal-direction allocation: parent records appended
};

struct SceneDev {
    Entry* buckets;
    int* bucket_next;
    Node* nodes;
    Voxel* voxels;
    unsigned long long* block_key;
    int* block_slot;
    uint8_t* block_fresh;
    unsigned long long* block_wmask;  // per block: 2x2x2-voxel sub-cubes holding a weighted voxel
    uint8_t* block_touched;           // instrumented renders: block read by a ray
    uint32_t* heap;
    unsigned long long* bindex;
    unsigned long long* dwm;
    uint32_t* sup;
    uint32_t* visible;
    float4* pix_world;   // per pixel of the current frame: T*p and |T*p - c| (-1 = invalid)
    uint32_t* pix_rgb;   // per pixel: r | g<<8 | b<<16
    // normal-direction allocation (VoxelScene.cu:768-912): per pool block the
    // parent pixel of the last normal ray that visited it, packed as
    // (frame + 1) << 32 | y << 16 | x (0 = none); cleared when the block is
    // claimed.  Integration reads a block's parent pixel instead of each
    // voxel's projection (VoxelScene.cu:1015-1035).
    unsigned long long* block_parent;
    unsigned long long* parent_key;  // this frame's (block, pixel) records from k_alloc
    uint32_t* parent_tag;            // y << 16 | x
    uint32_t parent_cap;
    int alloc_method;                // 1: camera-z band (Method 1), 2: camera + normal rays (Method 2)
    uint32_t frame_seq;              // frames integrated since reset (the parent tags' frame)
    SceneCounters* ctr;
    FrameCounters* frame;
    uint32_t num_buckets;
    int num_blocks;
    int max_nodes;
    int bidx_log2;  // k: toroidal block grid of 2^k positions per axis
    float voxel;
    float inv_voxel;  // RN(1 / voxel)
    bool div_fast;    // fixed-divisor division verified for this voxel size
    // [257]: entry d (1..256) = RN(1/d) when the one-correction quotient
    // (avg_div) equals IEEE division by d for every dividend, else 0 (IEEE
    // division); the running average divides by the new weight d
    const float* avg_recip;
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

// ------------------------------------------------ exact division shortcuts

// x / d for a running-average divisor d (the new weight, 1..256), given
// y = avg_recip[d]: one Markstein correction of the product x*y (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990): r = x - q d is exact and
// RN(q + r y) is the quotient.  For a fixed d the three operations commute
// with scaling x by a power of two while |x| stays in [2^-100, 2^100) (q, r
// and the result stay representable), and with negation, so the verification
// at scene creation over every x in [1, 2) covers that whole range; +0 gives
// +0 as IEEE division does.  Other x (and divisors that failed verification,
// y = 0) use IEEE division; -0 among them, which IEEE division keeps negative.
__device__ __forceinline__ float avg_div(float x, float d, float y) {
    const float ax = fabsf(x);
    if (y != 0.0f && ax < 0x1p100f && (ax >= 0x1p-100f || __float_as_uint(x) == 0u)) {
        const float q = __fmul_rn(x, y);
        const float r = __fmaf_rn(-q, d, x);
        return __fmaf_rn(r, y, q);
    }
    return x / d;
}

// For a camera distance w = RN(sqrt(.)) of a pixel's point: the smallest
// float D >= 0 with RN(sqrt(D)) >= w.  RN(sqrt(.)) is non-decreasing over
// the floats, so for every float D >= 0, RN(sqrt(D)) < w exactly when
// D < sqrt_threshold(w): integration decides the sign of a voxel's SDF
// (cameraDist < depthPos distance, VoxelScene.cu:1055-1066) on the squared
// distance without a square root per voxel.  w = +0, +inf and NaN are their
// own thresholds (the comparison is then false as with w itself).  The
// threshold is within a few ulps of RN(w*w); it is stepped there and checked
// against its definition, else found by bisection over the float order.
__device__ __forceinline__ float sqrt_threshold(float w) {
    if (!(w > 0.0f) || w == __int_as_float(0x7F800000)) return w;
    float c = w * w;
    bool ok = false;
    if (w >= 0x1p-60f && w <= 0x1p60f) {
        for (int i = 0; i < 8 && sqrtf(c) < w; ++i) c = __uint_as_float(__float_as_uint(c) + 1u);
        for (int i = 0; i < 8 && c > 0.0f && sqrtf(__uint_as_float(__float_as_uint(c) - 1u)) >= w; ++i)
            c = __uint_as_float(__float_as_uint(c) - 1u);
        ok = sqrtf(c) >= w && (c == 0.0f || sqrtf(__uint_as_float(__float_as_uint(c) - 1u)) < w);
    }
    if (!ok) {
        // min u in [0, +inf bits] with RN(sqrt(float(u))) >= w
        uint32_t lo = 0u, hi = 0x7F800000u;
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2u;
            if (sqrtf(__uint_as_float(mid)) >= w)
                hi = mid;
            else
                lo = mid + 1u;
        }
        c = __uint_as_float(lo);
    }
    return c;
}

// ------------------------------------------- sub-cube masks and skip grid

// 4x4x4 sub-cubes (2x2x2 voxels each) of a block: bit (cz*4 + cy)*4 + cx
constexpr unsigned long long kX0 = 0x1111111111111111ull, kX3 = 0x8888888888888888ull;
constexpr unsigned long long kY0 = 0x000F000F000F000Full, kY3 = 0xF000F000F000F000ull;
constexpr unsigned long long kZ0 = 0x000000000000FFFFull, kZ3 = 0xFFFF000000000000ull;

// Part of the one-sub-cube dilation of mask m that falls in the neighbour
// block at offset d (-1, 0, +1) along x / y / z.
__host__ __device__ __forceinline__ unsigned long long dil_x(unsigned long long m, int d) {
    return d == 0 ? (m | ((m & ~kX3) << 1) | ((m & ~kX0) >> 1)) : d > 0 ? ((m & kX3) >> 3) : ((m & kX0) << 3);
}
__host__ __device__ __forceinline__ unsigned long long dil_y(unsigned long long m, int d) {
    return d == 0 ? (m | ((m & ~kY3) << 4) | ((m & ~kY0) >> 4)) : d > 0 ? ((m & kY3) >> 12) : ((m & kY0) << 12);
}
__host__ __device__ __forceinline__ unsigned long long dil_z(unsigned long long m, int d) {
    return d == 0 ? (m | ((m & ~kZ3) << 16) | ((m & ~kZ0) >> 16)) : d > 0 ? ((m & kZ3) >> 48) : ((m & kZ0) << 48);
}

__host__ __device__ __forceinline__ uint32_t grid_bit(int x, int y, int z, int lg) {
    const uint32_t m = (1u << lg) - 1u;
    return (((uint32_t)z & m) << (2 * lg)) | (((uint32_t)y & m) << lg) | ((uint32_t)x & m);
}

// ------------------------------------------------------ dense block index

constexpr unsigned long long kIdxEmpty = 0xFFFFFFFFFFFFFFFFull;
constexpr unsigned long long kIdxShared = 0xFFFFFFFFFFFFFFFEull;
constexpr uint32_t kIdxPtrMask = 0x3FFFFFu;  // pools up to 2^22 - 3 blocks use the index

__host__ __device__ __forceinline__ uint32_t bidx_cell(int x, int y, int z, int k) {
    const uint32_t m = (1u << k) - 1u;
    return (((uint32_t)z & m) << (2 * k)) | (((uint32_t)y & m) << k) | ((uint32_t)x & m);
}

__host__ __device__ __forceinline__ unsigned long long bidx_tag(int x, int y, int z, int k) {
    const int hb = 21 - k;
    const unsigned long long m = (1ull << hb) - 1ull;
    return ((((unsigned long long)(unsigned)(x >> k)) & m) << (2 * hb)) |
           ((((unsigned long long)(unsigned)(y >> k)) & m) << hb) | (((unsigned long long)(unsigned)(z >> k)) & m);
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

// Pool index of block (x,y,z) through the dense index; the hash resolves
// cells shared by several blocks.  -1 = not allocated.
__device__ __forceinline__ int block_ptr(const SceneDev& s, int x, int y, int z) {
    if (!coord_ok(x, y, z)) return -1;
    const unsigned long long e = __ldg(s.bindex + bidx_cell(x, y, z, s.bidx_log2));
    if (e == kIdxEmpty) return -1;
    if (e == kIdxShared) return lookup_block(s, pack_key(x, y, z), x, y, z);
    return ((e >> 22) == bidx_tag(x, y, z, s.bidx_log2)) ? (int)(e & kIdxPtrMask) : -1;
}

__device__ __forceinline__ uint32_t pack_rgbw(uint32_t r, uint32_t g, uint32_t b, uint32_t w) {
    return r | (g << 8) | (b << 16) | (w << 24);
}

}  // namespace vsg
