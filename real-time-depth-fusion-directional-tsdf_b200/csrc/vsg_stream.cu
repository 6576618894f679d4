// vsg_stream.cu -- moving voxel blocks between a scene and host memory.
//
// Restates VoxelStreamingManager (VoxelStreamingManager.cu:36-84, 258-355,
// 443-714; VoxelStreamingManager.cpp:303-502, 836-1140):
//   stream out  every allocated block whose corner (8 b * voxel, computed as
//               the reference's int product times the float voxel size) lies
//               at distance >= radius from the centre leaves the scene: its
//               512 voxels are copied out, its hash entry is deleted and its
//               pool block returns to the free heap.  On the host the block
//               is filed in the chunk of worldToChunks(corner) (1 m chunks by
//               default, VoxelStreamingManager.cpp:905-922).
//   stream in   every stored chunk in the box of ceil(radius / extent)
//               chunks around the centre's chunk that passes isChunkInSphere
//               (:962-991) goes back: its blocks are inserted into the hash
//               and their voxels written to newly claimed pool blocks.
// B200 layout of the work: a selection kernel compacts candidate pool
// indices, an extraction kernel moves one block per warp (4 KiB of 16-byte
// loads per block, coalesced) and deletes it; insertion is one warp per
// block as well.  Transfers go through pinned staging in passes of up to
// 8192 blocks.
//
// Differences from the reference (its behaviour there is a defect, not a
// specification):
//   - stream-in inserts the blocks (the reference's insertion is switched
//     off, VoxelStreamingManager.cpp:575-579, so streamed-in data is lost);
//   - a block that is resident when its stored copy comes back, or that is
//     stored twice, is merged voxel by voxel with weights (merge_voxels) --
//     the reference would create a second hash entry for the same position;
//   - no 100,000-block cap per call and no grid bounds: every candidate goes
//     out (in passes) and blocks outside the 513^3-chunk grid are kept
//     instead of being dropped.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <new>
#include <atomic>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/vsg.h"
#include "vsg_device.cuh"
#include "vsg_fusion_core.cuh"
#include "vsg_internal.h"

namespace vsg {

constexpr uint32_t kStageBlocks = 8192;  // blocks per transfer pass (32 MiB of voxels)

struct StreamCounters {
    uint32_t found;   // stream-out candidates
    uint32_t merged;  // stream-in blocks merged into resident ones
    uint32_t failed;  // stream-in blocks that found no storage
    uint32_t pad;
};

struct StreamStage {
    int4* d_info = nullptr;
    Voxel* d_vox = nullptr;
    uint32_t* d_list = nullptr;
    StreamCounters* d_ctr = nullptr;
    int4* h_info = nullptr;
    Voxel* h_vox = nullptr;
};

// Per-voxel merge of two partial averages of one block position (no
// counterpart in the reference): weights add (capped at 255 like the
// integration's), SDF and colour are the weight-averaged values, colour
// truncated to 8 bits as integration does.
__host__ __device__ __forceinline__ Voxel merge_voxels(Voxel a, Voxel b) {
    const uint32_t wa = a.rgbw >> 24, wb = b.rgbw >> 24;
    if (wb == 0u) return a;
    if (wa == 0u) return b;
    const float fa = (float)wa, fb = (float)wb, fw = (float)(wa + wb);
    Voxel o;
    o.sdf = (a.sdf * fa + b.sdf * fb) / fw;
    uint32_t c[3];
    for (int i = 0; i < 3; ++i) {
        const float ca = (float)((a.rgbw >> (8 * i)) & 0xFFu), cb = (float)((b.rgbw >> (8 * i)) & 0xFFu);
        c[i] = (uint32_t)((ca * fa + cb * fb) / fw);
    }
    const uint32_t w = wa + wb > 255u ? 255u : wa + wb;
    o.rgbw = c[0] | (c[1] << 8) | (c[2] << 16) | (w << 24);
    return o;
}

namespace {

// SDFBlockToWorld (VoxelStreamingManager.cu:22-28): the int product
// coordinate * 8, converted, times the voxel size.
__host__ __device__ __forceinline__ float block_corner(int c, float v) { return (float)(c * kBlock) * v; }

__global__ void k_stream_select(SceneDev s, float cx, float cy, float cz, float radius, uint32_t* list, uint32_t cap,
                                StreamCounters* c) {
    const uint32_t hw = s.ctr->high_water;
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < hw; b += gridDim.x * blockDim.x) {
        const unsigned long long key = s.block_key[b];
        if (key == kKeyEmpty || key == kKeyTomb) continue;
        int x, y, z;
        unpack_key(key, x, y, z);
        // streamOutFindBlocksKernel_OPTIMIZED, VoxelStreamingManager.cu:56-69
        const float dx = block_corner(x, s.voxel) - cx;
        const float dy = block_corner(y, s.voxel) - cy;
        const float dz = block_corner(z, s.voxel) - cz;
        const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
        if (dist >= radius) {
            const uint32_t i = atomicAdd(&c->found, 1u);
            if (i < cap) list[i] = b;
        }
    }
}

// One warp per listed block: copy its voxels out, delete its hash entry and
// dense-index cell, return its pool block to the heap
// (streamOutCopyBlocksKernel, VoxelStreamingManager.cu:258-355).
__global__ void k_stream_extract(SceneDev s, const uint32_t* list, uint32_t n, int4* info, Voxel* out) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const uint32_t b = list[i];
        const uint4* src = reinterpret_cast<const uint4*>(s.voxels + (size_t)b * kVoxPerBlock);
        uint4* dst = reinterpret_cast<uint4*>(out + (size_t)i * kVoxPerBlock);
#pragma unroll
        for (int k = 0; k < 8; ++k) dst[k * 32 + lane] = src[k * 32 + lane];
        if (lane == 0) {
            const unsigned long long key = s.block_key[b];
            int x, y, z;
            unpack_key(key, x, y, z);
            info[i] = make_int4(x, y, z, (int)b);
            const int slot = s.block_slot[b];
            const int base = (int)s.num_buckets * kBucketSlots;
            if (slot < base)
                atomicExch(&s.buckets[slot].key, kKeyTomb);
            else
                atomicExch(&s.nodes[slot - base].key, kKeyTomb);
            if (b < kIdxPtrMask - 2u) {
                const unsigned long long mine = (bidx_tag(x, y, z, s.bidx_log2) << 22) | (unsigned long long)b;
                atomicCAS(s.bindex + bidx_cell(x, y, z, s.bidx_log2), mine, kIdxEmpty);
            }
            s.block_key[b] = kKeyEmpty;
            s.block_wmask[b] = 0ull;
            s.block_fresh[b] = 0;
            const int j = atomicAdd(&s.ctr->free_count, 1);
            s.heap[j] = b;
        }
    }
}

// lookup_block with volatile loads: sees entries inserted earlier in the
// same launch (the read-only path may not).
__device__ int lookup_block_fresh(const SceneDev& s, unsigned long long key, int x, int y, int z) {
    const uint32_t b = bucket_of(x, y, z, s.num_buckets);
    Entry* bk = s.buckets + (size_t)b * kBucketSlots;
    for (int j = 0; j < kBucketSlots; ++j) {
        const unsigned long long k = ld_volatile_u64(&bk[j].key);
        if (k == key) return ld_volatile_i32(&bk[j].ptr);
        if (k == kKeyEmpty) return -1;
    }
    int n = ld_volatile_i32(s.bucket_next + b);
    for (int it = 0; n >= 0 && it < s.max_nodes; ++it) {
        if (ld_volatile_u64(&s.nodes[n].key) == key) return ld_volatile_i32(&s.nodes[n].ptr);
        n = ld_volatile_i32(&s.nodes[n].next);
    }
    return -1;
}

// One warp per incoming block: insert (or find) its position, write or merge
// its voxels, then maintain the sub-cube weight mask and the ray-march skip
// grid exactly as integration does (streamInHashAllocKernel +
// streamInHashInitKernel, VoxelStreamingManager.cu:443-714).
__global__ void k_stream_insert(SceneDev s, const int4* info, const Voxel* in, uint32_t n, StreamCounters* c) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const int4 d = info[i];
        int ptr = -1, merged = 0;
        if (lane == 0) {
            if (coord_ok(d.x, d.y, d.z)) {
                const unsigned long long key = pack_key(d.x, d.y, d.z);
                ptr = lookup_block_fresh(s, key, d.x, d.y, d.z);
                if (ptr >= 0) {
                    merged = 1;
                } else {
                    insert_single(s, key, d.x, d.y, d.z, false);
                    ptr = lookup_block_fresh(s, key, d.x, d.y, d.z);
                }
                if (ptr < 0) atomicAdd(&c->failed, 1u);
            } else {
                atomicOr(&s.ctr->flags, (uint32_t)VSG_FLAG_COORD_RANGE);
                atomicAdd(&c->failed, 1u);
            }
        }
        ptr = __shfl_sync(0xFFFFFFFFu, ptr, 0);
        merged = __shfl_sync(0xFFFFFFFFu, merged, 0);
        if (ptr < 0) continue;
        Voxel* vb = s.voxels + (size_t)ptr * kVoxPerBlock;
        const Voxel* src = in + (size_t)i * kVoxPerBlock;
        const unsigned long long old_wm = merged ? s.block_wmask[ptr] : 0ull;
        unsigned long long wm = 0ull;
        const int lx = lane & 7;
#pragma unroll 4
        for (int k = 0; k < 16; ++k) {
            const int idx = k * 32 + lane;
            Voxel v = src[idx];
            if (merged) v = merge_voxels(vb[idx], v);
            vb[idx] = v;
            if (v.rgbw >> 24) {
                const int ly = (lane >> 3) + ((k & 1) << 2), lz = k >> 1;
                wm |= 1ull << ((((lz >> 1) * 4 + (ly >> 1)) * 4) + (lx >> 1));
            }
        }
        const unsigned wlo = __reduce_or_sync(0xFFFFFFFFu, (unsigned)wm);
        const unsigned whi = __reduce_or_sync(0xFFFFFFFFu, (unsigned)(wm >> 32));
        const unsigned long long nw = ((unsigned long long)whi << 32) | wlo;
        const unsigned long long newbits = nw & ~old_wm;
        if (newbits && lane < 27) {
            const int dx = lane % 3 - 1, dy = (lane / 3) % 3 - 1, dz = lane / 9 - 1;
            const unsigned long long mk = dil_z(dil_y(dil_x(newbits, dx), dy), dz);
            if (mk) {
                const int nx = d.x + dx, ny = d.y + dy, nz = d.z + dz;
                atomicOr(s.dwm + bidx_cell(nx, ny, nz, s.bidx_log2), mk);
                const uint32_t q = grid_bit(nx >> 3, ny >> 3, nz >> 3, s.bidx_log2 - 3);
                atomicOr(s.sup + (q >> 5), 1u << (q & 31));
            }
        }
        __syncwarp();
        if (lane == 0) {
            s.block_wmask[ptr] = old_wm | nw;
            s.block_fresh[ptr] = 0;
            if (merged) atomicAdd(&c->merged, 1u);
        }
    }
}

// ------------------------------------------------------------- host store

struct Coord3Hash {
    size_t operator()(const std::array<int, 3>& a) const {
        unsigned long long h = (unsigned long long)(unsigned)a[0] * 0x9E3779B97F4A7C15ull;
        h ^= (unsigned long long)(unsigned)a[1] * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
        h ^= (unsigned long long)(unsigned)a[2] * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};

}  // namespace

// Host voxel storage in slabs of kSlabBlocks blocks: appending a block
// copies its 4 KiB once (no regrowth of one large array), and slabs of
// chunks that stream back in return to the store's free list, so a long
// run stops faulting in fresh pages.
constexpr size_t kSlabBlocks = 16;

struct Chunk {
    std::vector<std::array<int, 3>> coords;
    std::vector<Voxel*> slabs;  // block i at slabs[i / kSlabBlocks] + (i % kSlabBlocks) * 512
    std::unordered_map<std::array<int, 3>, uint32_t, Coord3Hash> index;
    Voxel* block(size_t i) const { return slabs[i / kSlabBlocks] + (i % kSlabBlocks) * kVoxPerBlock; }
};

struct BlockStore {
    float ext[3] = {1.0f, 1.0f, 1.0f};
    float voxel = 0.0f;  // voxel size of the blocks held (0 = none yet)
    std::unordered_map<std::array<int, 3>, Chunk, Coord3Hash> chunks;
    uint64_t n_blocks = 0;
    std::vector<std::unique_ptr<Voxel[]>> slab_mem;  // every slab ever made (freed with the store)
    std::vector<Voxel*> free_slabs;

    Voxel* new_slab() {
        if (!free_slabs.empty()) {
            Voxel* s = free_slabs.back();
            free_slabs.pop_back();
            return s;
        }
        std::unique_ptr<Voxel[]> m(new Voxel[kSlabBlocks * kVoxPerBlock]);
        slab_mem.push_back(std::move(m));
        return slab_mem.back().get();
    }
    // drop a chunk, keeping its slabs for reuse
    void erase_chunk(const std::array<int, 3>& ck) {
        auto it = chunks.find(ck);
        if (it == chunks.end()) return;
        free_slabs.reserve(free_slabs.size() + it->second.slabs.size());
        n_blocks -= it->second.coords.size();
        for (Voxel* s : it->second.slabs) free_slabs.push_back(s);
        chunks.erase(it);
    }

    // worldToChunks, VoxelStreamingManager.cpp:905-922
    std::array<int, 3> chunk_of_world(const float p[3]) const {
        std::array<int, 3> c{};
        for (int i = 0; i < 3; ++i) {
            const float q = p[i] / ext[i];
            const float sg = (q > 0.0f) ? 1.0f : ((q < 0.0f) ? -1.0f : 0.0f);
            c[i] = static_cast<int>(q + sg * 0.5f);
        }
        return c;
    }
    // updateChunkGrid, :836-903: the chunk of the block's corner
    std::array<int, 3> chunk_of_block(int x, int y, int z, float v) const {
        const float p[3] = {block_corner(x, v), block_corner(y, v), block_corner(z, v)};
        return chunk_of_world(p);
    }
    // isChunkInSphere, :962-991 (its first test is implied by the second)
    bool chunk_in_sphere(const std::array<int, 3>& c, const float center[3], float radius) const {
        const float wx = (float)c[0] * ext[0], wy = (float)c[1] * ext[1], wz = (float)c[2] * ext[2];
        const float ce = std::max(std::max(ext[0], ext[1]), ext[2]);
        const float cr = 0.5f * ce * sqrtf(3.0f);
        const float dx = wx - center[0], dy = wy - center[1], dz = wz - center[2];
        const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
        return dist - cr <= radius;
    }

    void add(int x, int y, int z, const Voxel* v, float voxel_size) {
        add_to(chunks[chunk_of_block(x, y, z, voxel_size)], x, y, z, v, nullptr);
    }

    // File one block into its chunk; returns 1 when the block is new.  With
    // a lock, slabs are taken under it (chunk-parallel filing).  Every
    // allocation comes before the block is entered, so std::bad_alloc leaves
    // the chunk's blocks as they were (at most a spare slab is kept).
    int add_to(Chunk& ch, int x, int y, int z, const Voxel* v, std::mutex* lock) {
        const std::array<int, 3> key{x, y, z};
        auto it = ch.index.find(key);
        if (it != ch.index.end()) {
            Voxel* dst = ch.block(it->second);
            for (int i = 0; i < kVoxPerBlock; ++i) dst[i] = merge_voxels(dst[i], v[i]);
            return 0;
        }
        const size_t i = ch.coords.size();
        if (ch.coords.size() == ch.coords.capacity()) ch.coords.reserve(std::max<size_t>(16, 2 * i));
        if (i / kSlabBlocks >= ch.slabs.size()) {
            if (ch.slabs.size() == ch.slabs.capacity()) ch.slabs.reserve(std::max<size_t>(4, 2 * ch.slabs.size()));
            Voxel* slab;
            if (lock) {
                std::lock_guard<std::mutex> g(*lock);
                slab = new_slab();
            } else {
                slab = new_slab();
            }
            ch.slabs.push_back(slab);
        }
        ch.index.emplace(key, (uint32_t)i);
        ch.coords.push_back(key);
        std::memcpy(ch.block(i), v, kVoxPerBlock * sizeof(Voxel));
        if (!lock) ++n_blocks;
        return 1;
    }

    // File n blocks (stream-out pass): grouped by chunk, chunks filed in
    // parallel by up to 8 host threads (each chunk by one thread, so a
    // chunk's index and slab list need no lock; only the slab free list is
    // shared).  Same contents as n calls of add().
    void add_many(const int4* info, const Voxel* vox, uint32_t n, float voxel_size) {
        if (n < 512) {
            for (uint32_t i = 0; i < n; ++i) add(info[i].x, info[i].y, info[i].z, vox + (size_t)i * kVoxPerBlock,
                                                 voxel_size);
            return;
        }
        std::vector<std::pair<std::array<int, 3>, uint32_t>> keyed(n);
        for (uint32_t i = 0; i < n; ++i) keyed[i] = {chunk_of_block(info[i].x, info[i].y, info[i].z, voxel_size), i};
        std::stable_sort(keyed.begin(), keyed.end(),
                         [](const auto& a, const auto& b) { return a.first < b.first; });
        struct Group {
            Chunk* ch;
            uint32_t begin, end;
        };
        std::vector<Group> groups;
        for (uint32_t b = 0; b < n;) {
            uint32_t e = b + 1;
            while (e < n && keyed[e].first == keyed[b].first) ++e;
            groups.push_back({&chunks[keyed[b].first], b, e});  // element references survive rehashing
            b = e;
        }
        std::mutex lock;
        std::atomic<uint32_t> next{0};
        std::atomic<uint64_t> added{0};
        std::atomic<bool> out_of_memory{false};
        auto work = [&]() {
            uint64_t mine = 0;
            try {
                for (uint32_t g; (g = next.fetch_add(1)) < groups.size();)
                    for (uint32_t k = groups[g].begin; k < groups[g].end; ++k) {
                        const uint32_t i = keyed[k].second;
                        mine += (uint64_t)add_to(*groups[g].ch, info[i].x, info[i].y, info[i].z,
                                                 vox + (size_t)i * kVoxPerBlock, &lock);
                    }
            } catch (...) {  // host memory exhausted: stop every thread, report after the join
                out_of_memory = true;
                next = (uint32_t)groups.size();
            }
            added += mine;
        };
        const unsigned hw = std::thread::hardware_concurrency();
        const unsigned nt = std::min<unsigned>(std::min<unsigned>(hw ? hw : 1u, 8u), (unsigned)groups.size());
        std::vector<std::thread> pool;
        try {
            pool.reserve(nt);
            for (unsigned t = 1; t < nt; ++t) pool.emplace_back(work);
        } catch (...) {  // fewer threads: the ones started and this one take every group
        }
        work();
        for (auto& th : pool) th.join();
        n_blocks += added.load();
        if (out_of_memory) throw std::bad_alloc();
    }

    // streamInFindChunk, :993-1140: the chunks a stream-in takes (sorted,
    // so transfers are deterministic); radius < 0 takes every chunk.
    std::vector<std::array<int, 3>> chunks_for(const float center[3], float radius) const {
        std::vector<std::array<int, 3>> out;
        if (radius < 0.0f) {
            for (const auto& kv : chunks) out.push_back(kv.first);
        } else {
            const std::array<int, 3> cc = chunk_of_world(center);
            int cr[3];
            for (int i = 0; i < 3; ++i) cr[i] = static_cast<int>(std::ceil(radius / ext[i]));
            const double span = (2.0 * cr[0] + 1) * (2.0 * cr[1] + 1) * (2.0 * cr[2] + 1);
            if (span > 4.0 * (double)chunks.size() + 64.0) {
                // few stored chunks against a large box: test the stored ones
                for (const auto& kv : chunks) {
                    const auto& c = kv.first;
                    if (std::abs(c[0] - cc[0]) <= cr[0] && std::abs(c[1] - cc[1]) <= cr[1] &&
                        std::abs(c[2] - cc[2]) <= cr[2] && chunk_in_sphere(c, center, radius))
                        out.push_back(c);
                }
            } else {
                for (int x = cc[0] - cr[0]; x <= cc[0] + cr[0]; ++x)
                    for (int y = cc[1] - cr[1]; y <= cc[1] + cr[1]; ++y)
                        for (int z = cc[2] - cr[2]; z <= cc[2] + cr[2]; ++z) {
                            const std::array<int, 3> c{x, y, z};
                            if (chunks.count(c) && chunk_in_sphere(c, center, radius)) out.push_back(c);
                        }
            }
        }
        std::sort(out.begin(), out.end());
        return out;
    }
};

namespace {

int stage_for(Scene* sc, StreamStage** out) {
    if (!sc->stream_stage) {
        StreamStage* st = new (std::nothrow) StreamStage();
        if (!st) return VSG_ERR_OUT_OF_MEMORY;
        sc->stream_stage = st;
        const size_t nb = kStageBlocks;
        if (cudaMalloc(&st->d_info, nb * sizeof(int4)) != cudaSuccess ||
            cudaMalloc(&st->d_vox, nb * kVoxPerBlock * sizeof(Voxel)) != cudaSuccess ||
            cudaMalloc(&st->d_list, nb * sizeof(uint32_t)) != cudaSuccess ||
            cudaMalloc(&st->d_ctr, sizeof(StreamCounters)) != cudaSuccess ||
            cudaHostAlloc(&st->h_info, nb * sizeof(int4), cudaHostAllocDefault) != cudaSuccess ||
            cudaHostAlloc(&st->h_vox, nb * kVoxPerBlock * sizeof(Voxel), cudaHostAllocDefault) != cudaSuccess) {
            stream_stage_free(sc);
            return VSG_ERR_OUT_OF_MEMORY;
        }
    }
    *out = static_cast<StreamStage*>(sc->stream_stage);
    return VSG_OK;
}

int grid_for(const Scene* sc, uint32_t n) {  // one warp per block, 8 warps per CTA
    const long long want = ((long long)n + 7) / 8;
    const long long cap = (long long)sc->sm_count * 8;
    return (int)std::max(1ll, std::min(want, cap));
}

int read_counters(const StreamStage* st, StreamCounters* c, cudaStream_t s) {
    if (cudaMemcpyAsync(c, st->d_ctr, sizeof(*c), cudaMemcpyDeviceToHost, s) != cudaSuccess) return VSG_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return VSG_ERR_CUDA;
    return VSG_OK;
}

// Insert host blocks (coords + voxels) into the scene in staging passes.
int insert_blocks(Scene* sc, const std::vector<std::array<int, 3>>& coords, const std::vector<const Voxel*>& vox,
                  cudaStream_t st, uint32_t* n_merged, uint32_t* n_failed) {
    StreamStage* sg = nullptr;
    int rc = stage_for(sc, &sg);
    if (rc != VSG_OK) return rc;
    uint32_t merged = 0, failed = 0;
    for (size_t done = 0; done < coords.size();) {
        const uint32_t n = (uint32_t)std::min<size_t>(kStageBlocks, coords.size() - done);
        // gather into the pinned staging, contiguous ranges over up to 8 host threads
        auto gather = [&](uint32_t a, uint32_t b) {
            for (uint32_t i = a; i < b; ++i) {
                const auto& c = coords[done + i];
                sg->h_info[i] = make_int4(c[0], c[1], c[2], -1);
                std::memcpy(sg->h_vox + (size_t)i * kVoxPerBlock, vox[done + i], kVoxPerBlock * sizeof(Voxel));
            }
        };
        const unsigned hw = std::thread::hardware_concurrency();
        const unsigned nt = n < 512 ? 1u : std::min<unsigned>(hw ? hw : 1u, 8u);
        std::vector<std::thread> pool;
        unsigned started = 1;  // ranges 1 .. started-1 run on their own threads
        try {
            pool.reserve(nt);
            for (unsigned t = 1; t < nt; ++t, ++started)
                pool.emplace_back(gather, (uint32_t)((uint64_t)n * t / nt), (uint32_t)((uint64_t)n * (t + 1) / nt));
        } catch (...) {  // a thread could not start: this thread gathers the rest
        }
        gather(0, (uint32_t)((uint64_t)n / nt));
        if (started < nt) gather((uint32_t)((uint64_t)n * started / nt), n);
        for (auto& th : pool) th.join();
        if (cudaMemsetAsync(sg->d_ctr, 0, sizeof(StreamCounters), st) != cudaSuccess ||
            cudaMemcpyAsync(sg->d_info, sg->h_info, n * sizeof(int4), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(sg->d_vox, sg->h_vox, (size_t)n * kVoxPerBlock * sizeof(Voxel), cudaMemcpyHostToDevice,
                            st) != cudaSuccess)
            return VSG_ERR_CUDA;
        k_stream_insert<<<grid_for(sc, n), 256, 0, st>>>(sc->dev, sg->d_info, sg->d_vox, n, sg->d_ctr);
        if (cudaGetLastError() != cudaSuccess) return VSG_ERR_CUDA;
        StreamCounters c{};
        rc = read_counters(sg, &c, st);  // also frees the pinned staging for the next pass
        if (rc != VSG_OK) return rc;
        merged += c.merged;
        failed += c.failed;
        done += n;
    }
    if (n_merged) *n_merged = merged;
    if (n_failed) *n_failed = failed;
    return VSG_OK;
}

}  // namespace

void stream_stage_free(Scene* sc) {
    StreamStage* st = static_cast<StreamStage*>(sc->stream_stage);
    if (!st) return;
    cudaFree(st->d_info);
    cudaFree(st->d_vox);
    cudaFree(st->d_list);
    cudaFree(st->d_ctr);
    cudaFreeHost(st->h_info);
    cudaFreeHost(st->h_vox);
    delete st;
    sc->stream_stage = nullptr;
}

}  // namespace vsg

struct vsg_block_store {
    vsg::BlockStore impl;
};

namespace {

// Checkpoint file: the reference's streaming records (VoxelStreamingManager.h:
// 30-76): SDFBlockInfo {int3 pos, int ptr} then SDFBlock {512 x VoxelData
// {uchar3 color, uchar weight, float sdf, uchar isUpdated, uchar
// isZeroCrossing, 2 pad}}, after a 32-byte header.
constexpr char kMagic[8] = {'V', 'S', 'G', 'B', 'L', 'K', '0', '1'};
struct FileHeader {
    char magic[8];
    uint32_t info_bytes;   // 16
    uint32_t voxel_bytes;  // 12
    uint64_t n_blocks;
    float voxel_size;
    uint32_t reserved;
};
static_assert(sizeof(FileHeader) == 32, "header layout");

void to_ref_voxel(const vsg::Voxel& v, unsigned char o[12]) {
    o[0] = (unsigned char)(v.rgbw & 0xFFu);
    o[1] = (unsigned char)((v.rgbw >> 8) & 0xFFu);
    o[2] = (unsigned char)((v.rgbw >> 16) & 0xFFu);
    o[3] = (unsigned char)(v.rgbw >> 24);
    std::memcpy(o + 4, &v.sdf, 4);
    o[8] = o[9] = o[10] = o[11] = 0;
}

vsg::Voxel from_ref_voxel(const unsigned char o[12]) {
    vsg::Voxel v;
    std::memcpy(&v.sdf, o + 4, 4);
    v.rgbw = (uint32_t)o[0] | ((uint32_t)o[1] << 8) | ((uint32_t)o[2] << 16) | ((uint32_t)o[3] << 24);
    return v;
}

int write_blocks(const char* path, float voxel, const std::vector<std::array<int, 3>>& coords,
                 const std::vector<const vsg::Voxel*>& vox) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return VSG_ERR_INVALID_ARG;
    FileHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.info_bytes = 16;
    h.voxel_bytes = 12;
    h.n_blocks = coords.size();
    h.voxel_size = voxel;
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
    for (size_t i = 0; ok && i < coords.size(); ++i) {
        const int32_t rec[4] = {coords[i][0], coords[i][1], coords[i][2], -1};
        ok = std::fwrite(rec, sizeof(rec), 1, f) == 1;
    }
    std::vector<unsigned char> buf(vsg::kVoxPerBlock * 12);
    for (size_t i = 0; ok && i < coords.size(); ++i) {
        for (int v = 0; v < vsg::kVoxPerBlock; ++v) to_ref_voxel(vox[i][v], buf.data() + 12 * v);
        ok = std::fwrite(buf.data(), buf.size(), 1, f) == 1;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? VSG_OK : VSG_ERR_INVALID_ARG;
}

int read_blocks(const char* path, float* voxel, std::vector<std::array<int, 3>>* coords,
                std::vector<vsg::Voxel>* vox) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return VSG_ERR_INVALID_ARG;
    FileHeader h{};
    bool ok = std::fread(&h, sizeof(h), 1, f) == 1 && std::memcmp(h.magic, kMagic, 8) == 0 && h.info_bytes == 16 &&
              h.voxel_bytes == 12 && h.n_blocks < (1ull << 32);
    // the header's block count must be the one the file holds: a truncated or
    // corrupted file is refused before any buffer is sized from the count
    if (ok) {
        std::error_code ec;
        const uintmax_t size = std::filesystem::file_size(path, ec);
        ok = !ec && size == sizeof(FileHeader) + h.n_blocks * (16u + 12u * (uint64_t)vsg::kVoxPerBlock);
    }
    if (ok) {
        coords->resize(h.n_blocks);
        vox->resize(h.n_blocks * vsg::kVoxPerBlock);
        for (uint64_t i = 0; ok && i < h.n_blocks; ++i) {
            int32_t rec[4];
            ok = std::fread(rec, sizeof(rec), 1, f) == 1;
            (*coords)[i] = {rec[0], rec[1], rec[2]};
        }
        std::vector<unsigned char> buf(vsg::kVoxPerBlock * 12);
        for (uint64_t i = 0; ok && i < h.n_blocks; ++i) {
            ok = std::fread(buf.data(), buf.size(), 1, f) == 1;
            for (int v = 0; ok && v < vsg::kVoxPerBlock; ++v)
                (*vox)[i * vsg::kVoxPerBlock + v] = from_ref_voxel(buf.data() + 12 * v);
        }
        *voxel = h.voxel_size;
    }
    std::fclose(f);
    return ok ? VSG_OK : VSG_ERR_INVALID_ARG;
}

bool scene_on_current_device(const vsg_scene* s) {
    int dev = -1;
    cudaGetDevice(&dev);
    return dev == s->impl.device;
}

int free_pool_blocks(vsg::Scene* sc, cudaStream_t st, uint64_t* out) {
    vsg::SceneCounters ctr{};
    if (cudaMemcpyAsync(&ctr, sc->dev.ctr, sizeof(ctr), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return VSG_ERR_CUDA;
    *out = (uint64_t)std::max(ctr.free_count, 0);
    return VSG_OK;
}

}  // namespace

extern "C" {

int vsg_store_create(const float chunk_extent[3], vsg_block_store** out) {
    if (!out) return VSG_ERR_INVALID_ARG;
    *out = nullptr;
    float e[3] = {1.0f, 1.0f, 1.0f};  // g_streamingVoxelExtents, globalParamasConfig.cpp:124
    if (chunk_extent)
        for (int i = 0; i < 3; ++i) {
            if (!(chunk_extent[i] > 0.0f) || !std::isfinite(chunk_extent[i])) return VSG_ERR_INVALID_ARG;
            e[i] = chunk_extent[i];
        }
    vsg_block_store* st = new (std::nothrow) vsg_block_store();
    if (!st) return VSG_ERR_OUT_OF_MEMORY;
    std::memcpy(st->impl.ext, e, sizeof(e));
    *out = st;
    return VSG_OK;
}

int vsg_store_destroy(vsg_block_store* st) {
    if (!st) return VSG_ERR_INVALID_ARG;
    delete st;
    return VSG_OK;
}

int vsg_store_info(const vsg_block_store* st, uint64_t* n_blocks, uint64_t* n_chunks) {
    if (!st) return VSG_ERR_INVALID_ARG;
    if (n_blocks) *n_blocks = st->impl.n_blocks;
    if (n_chunks) *n_chunks = st->impl.chunks.size();
    return VSG_OK;
}

int vsg_store_count(const vsg_block_store* st, const float center[3], float radius, uint64_t* n_blocks,
                    uint64_t* n_chunks) {
    return vsg::host_guard([&]() -> int {
        if (!st || (!center && radius >= 0.0f)) return VSG_ERR_INVALID_ARG;
        const float zero[3] = {0.0f, 0.0f, 0.0f};
        const std::vector<std::array<int, 3>> take = st->impl.chunks_for(center ? center : zero, radius);
        uint64_t nb = 0;
        for (const auto& ck : take) nb += st->impl.chunks.at(ck).coords.size();
        if (n_blocks) *n_blocks = nb;
        if (n_chunks) *n_chunks = take.size();
        return VSG_OK;
    });
}

int vsg_store_add_records(vsg_block_store* st, float voxel_size, const int32_t* infos, const uint8_t* voxels,
                          uint64_t n) {
    return vsg::host_guard([&]() -> int {
        if (!st || !(voxel_size > 0.0f) || (n && (!infos || !voxels))) return VSG_ERR_INVALID_ARG;
        if (n == 0) return VSG_OK;
        if (st->impl.n_blocks && st->impl.voxel != voxel_size) return VSG_ERR_INVALID_ARG;
        st->impl.voxel = voxel_size;
        // converted and filed in passes of up to 8192 blocks (add_many: chunk-parallel,
        // repeats merged in input order)
        const uint64_t pass = std::min<uint64_t>(n, 8192);
        std::vector<int4> info((size_t)pass);
        std::vector<vsg::Voxel> blk((size_t)pass * vsg::kVoxPerBlock);
        for (uint64_t done = 0; done < n;) {
            const uint32_t m = (uint32_t)std::min<uint64_t>(pass, n - done);
            for (uint32_t j = 0; j < m; ++j) {
                const uint64_t i = done + j;
                info[j] = make_int4(infos[4 * i], infos[4 * i + 1], infos[4 * i + 2], -1);
                const uint8_t* src = voxels + i * (uint64_t)vsg::kVoxPerBlock * 12u;
                for (int v = 0; v < vsg::kVoxPerBlock; ++v)
                    blk[(size_t)j * vsg::kVoxPerBlock + v] = from_ref_voxel(src + 12 * v);
            }
            st->impl.add_many(info.data(), blk.data(), m, voxel_size);
            done += m;
        }
        return VSG_OK;
    });
}

int vsg_store_export(const vsg_block_store* st, int32_t* coords, uint8_t* voxels, uint64_t max_blocks,
                     uint64_t* n_out) {
    return vsg::host_guard([&]() -> int {
        if (!st || !n_out) return VSG_ERR_INVALID_ARG;
        *n_out = st->impl.n_blocks;
        if (st->impl.n_blocks > max_blocks) return VSG_ERR_TOO_LARGE;
        if (!coords) return VSG_ERR_INVALID_ARG;
        std::vector<std::pair<std::array<int, 3>, const vsg::Voxel*>> all;
        all.reserve(st->impl.n_blocks);
        for (const auto& kv : st->impl.chunks)
            for (size_t i = 0; i < kv.second.coords.size(); ++i)
                all.push_back({kv.second.coords[i], kv.second.block(i)});
        std::sort(all.begin(), all.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (size_t i = 0; i < all.size(); ++i) {
            coords[3 * i + 0] = all[i].first[0];
            coords[3 * i + 1] = all[i].first[1];
            coords[3 * i + 2] = all[i].first[2];
            if (voxels) std::memcpy(voxels + i * vsg::kVoxPerBlock * 8, all[i].second, vsg::kVoxPerBlock * 8);
        }
        return VSG_OK;
    });
}

int vsg_store_save(const vsg_block_store* st, const char* path) {
    return vsg::host_guard([&]() -> int {
        if (!st || !path) return VSG_ERR_INVALID_ARG;
        std::vector<std::array<int, 3>> coords;
        std::vector<const vsg::Voxel*> vox;
        for (const auto& kv : st->impl.chunks)
            for (size_t i = 0; i < kv.second.coords.size(); ++i) {
                coords.push_back(kv.second.coords[i]);
                vox.push_back(kv.second.block(i));
            }
        return write_blocks(path, st->impl.voxel, coords, vox);
    });
}

int vsg_store_load(vsg_block_store* st, const char* path) {
    return vsg::host_guard([&]() -> int {
        if (!st || !path) return VSG_ERR_INVALID_ARG;
        float voxel = 0.0f;
        std::vector<std::array<int, 3>> coords;
        std::vector<vsg::Voxel> vox;
        const int rc = read_blocks(path, &voxel, &coords, &vox);
        if (rc != VSG_OK) return rc;
        if (coords.empty()) return VSG_OK;
        if (st->impl.n_blocks && st->impl.voxel != voxel) return VSG_ERR_INVALID_ARG;
        st->impl.voxel = voxel;
        for (size_t i = 0; i < coords.size(); ++i)
            st->impl.add(coords[i][0], coords[i][1], coords[i][2], vox.data() + i * vsg::kVoxPerBlock, voxel);
        return VSG_OK;
    });
}

int vsg_stream_out(vsg_scene* s, vsg_block_store* store, const float center[3], float radius, uint32_t* n_out,
                   vsg_stream_t stream) {
    return vsg::host_guard([&]() -> int {
        if (!s || !store || !center || !scene_on_current_device(s)) return VSG_ERR_INVALID_ARG;
        vsg::Scene* sc = &s->impl;
        const float voxel = sc->params.voxel_size;
        if (store->impl.n_blocks && store->impl.voxel != voxel) return VSG_ERR_INVALID_ARG;
        vsg::StreamStage* sg = nullptr;
        int rc = vsg::stage_for(sc, &sg);
        if (rc != VSG_OK) return rc;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        uint32_t total = 0;
        for (;;) {
            if (cudaMemsetAsync(sg->d_ctr, 0, sizeof(vsg::StreamCounters), st) != cudaSuccess) return VSG_ERR_CUDA;
            vsg::k_stream_select<<<sc->sm_count * 4, 256, 0, st>>>(sc->dev, center[0], center[1], center[2], radius,
                                                                   sg->d_list, vsg::kStageBlocks, sg->d_ctr);
            if (cudaGetLastError() != cudaSuccess) return VSG_ERR_CUDA;
            vsg::StreamCounters c{};
            rc = vsg::read_counters(sg, &c, st);
            if (rc != VSG_OK) return rc;
            const uint32_t n = std::min(c.found, vsg::kStageBlocks);
            if (n == 0) break;
            vsg::k_stream_extract<<<vsg::grid_for(sc, n), 256, 0, st>>>(sc->dev, sg->d_list, n, sg->d_info, sg->d_vox);
            if (cudaGetLastError() != cudaSuccess ||
                cudaMemcpyAsync(sg->h_info, sg->d_info, n * sizeof(int4), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaMemcpyAsync(sg->h_vox, sg->d_vox, (size_t)n * vsg::kVoxPerBlock * sizeof(vsg::Voxel),
                                cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                return VSG_ERR_CUDA;
            store->impl.voxel = voxel;
            store->impl.add_many(sg->h_info, sg->h_vox, n, voxel);
            total += n;
            if (c.found <= vsg::kStageBlocks) break;
        }
        if (n_out) *n_out = total;
        return VSG_OK;
    });
}

int vsg_stream_in(vsg_scene* s, vsg_block_store* store, const float center[3], float radius, uint32_t* n_in,
                  uint32_t* n_merged, vsg_stream_t stream) {
    return vsg::host_guard([&]() -> int {
        if (!s || !store || (!center && radius >= 0.0f) || !scene_on_current_device(s)) return VSG_ERR_INVALID_ARG;
        vsg::Scene* sc = &s->impl;
        vsg::BlockStore& bs = store->impl;
        if (n_in) *n_in = 0;
        if (n_merged) *n_merged = 0;
        if (bs.n_blocks == 0) return VSG_OK;
        if (bs.voxel != sc->params.voxel_size) return VSG_ERR_INVALID_ARG;
        const float zero[3] = {0.0f, 0.0f, 0.0f};
        const std::vector<std::array<int, 3>> take = bs.chunks_for(center ? center : zero, radius);
        std::vector<std::array<int, 3>> coords;
        std::vector<const vsg::Voxel*> vox;
        for (const auto& ck : take) {
            const vsg::Chunk& ch = bs.chunks.at(ck);
            for (size_t i = 0; i < ch.coords.size(); ++i) {
                coords.push_back(ch.coords[i]);
                vox.push_back(ch.block(i));
            }
        }
        if (coords.empty()) return VSG_OK;
        // the pool must hold every incoming block (a merge needs none, so the
        // test is conservative); otherwise nothing moves
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        uint64_t free_blocks = 0;
        int rc = free_pool_blocks(sc, st, &free_blocks);
        if (rc != VSG_OK) return rc;
        if (free_blocks < coords.size()) return VSG_ERR_TOO_LARGE;
        uint32_t merged = 0, failed = 0;
        rc = vsg::insert_blocks(sc, coords, vox, st, &merged, &failed);
        if (rc != VSG_OK) return rc;
        for (const auto& ck : take) {
            bs.erase_chunk(ck);
        }
        if (n_in) *n_in = (uint32_t)coords.size() - failed;
        if (n_merged) *n_merged = merged;
        return failed ? VSG_ERR_OUT_OF_MEMORY : VSG_OK;
    });
}

int vsg_scene_save(vsg_scene* s, const char* path) {
    return vsg::host_guard([&]() -> int {
        if (!s || !path) return VSG_ERR_INVALID_ARG;
        uint32_t n = 0;
        int32_t dummy[3];
        int rc = vsg_scene_export(s, dummy, nullptr, 0, &n);
        if (rc != VSG_OK && rc != VSG_ERR_TOO_LARGE) return rc;
        std::vector<int32_t> c((size_t)n * 3 + 3);
        std::vector<vsg::Voxel> v((size_t)n * vsg::kVoxPerBlock + 1);
        rc = vsg_scene_export(s, c.data(), reinterpret_cast<uint8_t*>(v.data()), n, &n);
        if (rc != VSG_OK) return rc;
        std::vector<std::array<int, 3>> coords(n);
        std::vector<const vsg::Voxel*> vox(n);
        for (uint32_t i = 0; i < n; ++i) {
            coords[i] = {c[3 * i], c[3 * i + 1], c[3 * i + 2]};
            vox[i] = v.data() + (size_t)i * vsg::kVoxPerBlock;
        }
        return write_blocks(path, s->impl.params.voxel_size, coords, vox);
    });
}

int vsg_scene_load(vsg_scene* s, const char* path, vsg_stream_t stream) {
    return vsg::host_guard([&]() -> int {
        if (!s || !path || !scene_on_current_device(s)) return VSG_ERR_INVALID_ARG;
        float voxel = 0.0f;
        std::vector<std::array<int, 3>> coords;
        std::vector<vsg::Voxel> vox;
        int rc = read_blocks(path, &voxel, &coords, &vox);
        if (rc != VSG_OK) return rc;
        if (coords.empty()) return VSG_OK;
        if (voxel != s->impl.params.voxel_size) return VSG_ERR_INVALID_ARG;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        uint64_t free_blocks = 0;
        rc = free_pool_blocks(&s->impl, st, &free_blocks);
        if (rc != VSG_OK) return rc;
        if (free_blocks < coords.size()) return VSG_ERR_TOO_LARGE;
        std::vector<const vsg::Voxel*> ptrs(coords.size());
        for (size_t i = 0; i < coords.size(); ++i) ptrs[i] = vox.data() + i * vsg::kVoxPerBlock;
        uint32_t failed = 0;
        rc = vsg::insert_blocks(&s->impl, coords, ptrs, st, nullptr, &failed);
        if (rc != VSG_OK) return rc;
        return failed ? VSG_ERR_OUT_OF_MEMORY : VSG_OK;
    });
}

}  // extern "C"
