// vsg_fusion_core.cuh -- device code of allocation, visible-block selection
// and integration, shared by the per-scene kernels (vsg_fusion.cu) and the
// batched kernels (vsg_batch.cu).  The per-CTA entry points are
//   alloc_tile      one 16x16 pixel tile
//   select_blocks   a strided range of one scene's pool blocks
//   integrate_work  warps draining one scene's visible-block list
#pragma once

#include <cuda_runtime.h>

#include "../../include/vsg.h"
#include "vsg_device.cuh"

namespace vsg {

constexpr int kTile = 16;        // pixels per CTA side
constexpr int kSetCap = 1024;    // shared-memory de-duplication set
constexpr int kMaxDDA = 1024;    // VoxelScene.cu:417

struct AllocArgs {
    SceneDev s;
    const float* pm;
    const uint8_t* rgb;
    const float* nm;  // camera-space normals (normal-direction allocation only)
    int W, H;
    float trunc;
    Pose pose;
};

// worldToSDFBlock, VoxelScene.cu:74-96 (truncating conversion).
static __device__ __forceinline__ void world_to_block_alloc(float px, float py, float pz, float v, int& bx, int& by,
                                                     int& bz) {
    float q[3] = {px / v, py / v, pz / v};
    int o[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float sg = (q[a] > 0) ? 1.0f : ((q[a] < 0) ? -1.0f : 0.0f);
        int iv = __float2int_rz(q[a] + sg * 0.5f);
        if (iv < 0) iv = (int)((unsigned)iv - 7u);
        o[a] = iv / kBlock;
    }
    bx = o[0];
    by = o[1];
    bz = o[2];
}

static __device__ __forceinline__ void xform(const Pose& P, float x, float y, float z, float& ox, float& oy,
                                      float& oz) {
    ox = P.T[0] * x + P.T[1] * y + P.T[2] * z + P.T[3];
    oy = P.T[4] * x + P.T[5] * y + P.T[6] * z + P.T[7];
    oz = P.T[8] * x + P.T[9] * y + P.T[10] * z + P.T[11];
}

// Give a freshly inserted key storage.  entry_key / entry_ptr are the
// fields of the slot (bucket entry or chain node) the caller now owns.
// Heap pop as consumeHeap in VoxelScene.cu:183-195 (reference pops index
// heapCounter, we pop free_count - 1: the same stack).  from_frame: the
// block comes from a frame's allocation (counted as new this frame);
// blocks streamed back in from host memory are not.
static __device__ __noinline__ bool claim_block(const SceneDev& s, unsigned long long key, unsigned long long* entry_key,
                            int* entry_ptr, int slot_index, bool from_frame = true) {
    int old = atomicSub(&s.ctr->free_count, 1);
    if (old <= 0) {
        atomicAdd(&s.ctr->free_count, 1);
        atomicExch(entry_key, kKeyTomb);
        atomicOr(&s.ctr->flags, (uint32_t)VSG_FLAG_HEAP_EXHAUSTED);
        atomicAdd(&s.ctr->alloc_fail, 1u);
        return false;
    }
    const uint32_t blk = s.heap[old - 1];
    *entry_ptr = (int)blk;
    s.block_key[blk] = key;
    s.block_slot[blk] = slot_index;
    s.block_fresh[blk] = 1;
    s.block_parent[blk] = 0ull;
    atomicMax(&s.ctr->high_water, blk + 1);
    int x, y, z;
    unpack_key(key, x, y, z);
    // dense index: first block of a cell owns it, a second one marks it shared
    {
        unsigned long long* cell = s.bindex + bidx_cell(x, y, z, s.bidx_log2);
        const unsigned long long mine = blk < kIdxPtrMask - 2u
                                            ? ((bidx_tag(x, y, z, s.bidx_log2) << 22) | (unsigned long long)blk)
                                            : kIdxShared;
        const unsigned long long prev = atomicCAS(cell, kIdxEmpty, mine);
        if (prev != kIdxEmpty && prev != mine && prev != kIdxShared) atomicExch(cell, kIdxShared);
    }
    if (from_frame) atomicAdd(&s.frame->n_new, 1u);
    return true;
}

// Search the overflow chain of bucket b for key; append it when absent.
// Lock-free: a node is published by CAS on the tail link.
static __device__ __noinline__ void chain_insert(const SceneDev& s, uint32_t b, unsigned long long key, bool insert,
                                                 bool from_frame = true) {
    int* link = s.bucket_next + b;
    int mine = -1;
    const int base = (int)s.num_buckets * kBucketSlots;
    for (int it = 0; it <= s.max_nodes + 1; ++it) {
        int n = ld_volatile_i32(link);
        if (n < 0) {
            if (!insert) return;
            if (mine < 0) {
                mine = atomicAdd(&s.ctr->nodes_used, 1);
                if (mine >= s.max_nodes) {
                    atomicOr(&s.ctr->flags, (uint32_t)VSG_FLAG_CHAIN_EXHAUSTED);
                    atomicAdd(&s.ctr->alloc_fail, 1u);
                    return;
                }
                s.nodes[mine].ptr = -1;
                s.nodes[mine].next = -1;
                s.nodes[mine].key = key;
                __threadfence();
            }
            int prev = atomicCAS(link, -1, mine);
            if (prev == -1) {
                claim_block(s, key, &s.nodes[mine].key, &s.nodes[mine].ptr, base + mine, from_frame);
                return;
            }
            n = prev;
        }
        if (ld_volatile_u64(&s.nodes[n].key) == key) {
            if (mine >= 0) s.nodes[mine].key = kKeyTomb;  // unpublished spare
            return;
        }
        link = &s.nodes[n].next;
    }
    atomicOr(&s.ctr->flags, (uint32_t)VSG_FLAG_INSERT_RETRY);
}

static __device__ bool chain_contains(const SceneDev& s, uint32_t b, unsigned long long key) {
    int n = ld_volatile_i32(s.bucket_next + b);
    for (int it = 0; n >= 0 && it < s.max_nodes; ++it) {
        if (ld_volatile_u64(&s.nodes[n].key) == key) return true;
        n = ld_volatile_i32(&s.nodes[n].next);
    }
    return false;
}

// Single-thread insert (fallback when the shared set overflows).
static __device__ __noinline__ void insert_single(const SceneDev& s, unsigned long long key, int x, int y, int z,
                                                  bool from_frame = true) {
    const uint32_t b = bucket_of(x, y, z, s.num_buckets);
    Entry* bk = s.buckets + (size_t)b * kBucketSlots;
    for (int it = 0; it < 4 * kBucketSlots; ++it) {
        int first = -1;
        unsigned long long seen = 0;
        bool found = false;
        for (int j = 0; j < kBucketSlots; ++j) {
            unsigned long long k = ld_volatile_u64(&bk[j].key);
            if (k == key) {
                found = true;
                break;
            }
            if (first < 0 && (k == kKeyEmpty || k == kKeyTomb)) {
                first = j;
                seen = k;
            }
            if (k == kKeyEmpty) break;
        }
        if (found) return;
        if (first < 0) {
            chain_insert(s, b, key, true, from_frame);
            return;
        }
        if (seen == kKeyTomb && chain_contains(s, b, key)) return;
        unsigned long long prev = atomicCAS(&bk[first].key, seen, key);
        if (prev == seen) {
            claim_block(s, key, &bk[first].key, &bk[first].ptr, (int)(b * kBucketSlots + first), from_frame);
            return;
        }
    }
    atomicOr(&s.ctr->flags, (uint32_t)VSG_FLAG_INSERT_RETRY);
}

// Warp-cooperative insert of up to 4 keys (one per 8-lane group).  Lane j of
// a group reads slot j of the key's bucket; ballots find a match or the
// first free slot, whose lane issues the CAS.  A bucket slot only goes from
// free to used while allocation runs, so everyone racing on one key ends at
// the same first free slot.  All lanes of the warp must call this.
static __device__ void coop_insert(const SceneDev& s, unsigned long long key, bool active) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 3, sub = lane & 7;
    int x = 0, y = 0, z = 0;
    if (active) unpack_key(key, x, y, z);
    const uint32_t b = active ? bucket_of(x, y, z, s.num_buckets) : 0u;
    Entry* bk = s.buckets + (size_t)b * kBucketSlots;
    bool pending = active;
    for (int it = 0; it < 4 * kBucketSlots; ++it) {
        if (!__any_sync(0xFFFFFFFFu, pending)) return;
        unsigned long long cur = pending ? ld_volatile_u64(&bk[sub].key) : 0ull;
        const unsigned mm = __ballot_sync(0xFFFFFFFFu, pending && cur == key);
        const unsigned fm = __ballot_sync(0xFFFFFFFFu, pending && (cur == kKeyEmpty || cur == kKeyTomb));
        const unsigned gm = (mm >> (g * 8)) & 0xFFu;
        const unsigned gf = (fm >> (g * 8)) & 0xFFu;
        const int lead = gf ? (__ffs(gf) - 1) : 0;
        int res = 0;  // 1 = done
        if (pending) {
            if (gm) {
                res = 1;
            } else if (!gf) {
                if (sub == 0) chain_insert(s, b, key, true);
                res = 1;
            } else if (sub == lead) {
                if (cur == kKeyTomb && chain_contains(s, b, key)) {
                    res = 1;
                } else {
                    unsigned long long prev = atomicCAS(&bk[lead].key, cur, key);
                    if (prev == cur) {
                        claim_block(s, key, &bk[lead].key, &bk[lead].ptr, (int)(b * kBucketSlots + lead));
                        res = 1;
                    }
                }
            }
        }
        const int r = __shfl_sync(0xFFFFFFFFu, res, (g * 8) + lead);
        if (pending && (gm || !gf || r)) pending = false;
    }
    if (pending && sub == 0) atomicOr(&s.ctr->flags, (uint32_t)VSG_FLAG_INSERT_RETRY);
}

// Slot of k in the tile's shared set (inserted when absent), or -1 when
// the probe gives up (the set is full).
static __device__ __forceinline__ int set_insert(unsigned long long* set, unsigned long long k) {
    uint32_t h = (uint32_t)((k * 0x9E3779B97F4A7C15ull) >> 54) & (kSetCap - 1);
#pragma unroll 1
    for (int p = 0; p < 32; ++p) {
        unsigned long long cur = *(volatile unsigned long long*)(set + h);
        if (cur == k) return (int)h;
        if (cur == kKeyEmpty) {
            unsigned long long prev = atomicCAS(set + h, kKeyEmpty, k);
            if (prev == kKeyEmpty || prev == k) return (int)h;
        }
        h = (h + 1) & (kSetCap - 1);
    }
    return -1;
}

// A (block, parent pixel) record for apply_parents.
static __device__ __forceinline__ void append_parent(const SceneDev& s, unsigned long long key, uint32_t tag) {
    const uint32_t i = atomicAdd(&s.frame->n_parent, 1u);
    if (i < s.parent_cap) {
        s.parent_key[i] = key;
        s.parent_tag[i] = tag;
    } else {
        atomicOr(&s.ctr->flags, (uint32_t)VSG_FLAG_PARENT_OVERFLOW);
    }
}

// allocateBlocksAlongRay, VoxelScene.cu:295-481: nothing when both ends
// fall in one block (:345-348); else a block-level DDA from st to en with
// boundaries at (id + [step > 0]) * 8v - v/2 (:373-394), x only when its
// tMax is strictly smallest, then y when tMax.y < tMax.z, else z
// (:464-475), at most 1024 blocks (:417).  Visited blocks go into the
// tile's set, or straight into the table when the set is full.  ptag != 0
// (normal rays): (y << 16 | x) + 1 of the pixel, kept as the maximum per
// set slot.
static __device__ void dda_ray(const SceneDev& s, unsigned long long* set, uint32_t* set_tag, const float st[3],
                               const float en[3], uint32_t ptag) {
    const float v = s.voxel;
    int c[3], e[3];
    world_to_block_alloc(st[0], st[1], st[2], v, c[0], c[1], c[2]);
    world_to_block_alloc(en[0], en[1], en[2], v, e[0], e[1], e[2]);
    if (c[0] == e[0] && c[1] == e[1] && c[2] == e[2]) return;
    float d[3] = {en[0] - st[0], en[1] - st[1], en[2] - st[2]};
    const float len = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (len < 1e-6f) return;
    d[0] /= len;
    d[1] /= len;
    d[2] /= len;
    const float ext = (float)kBlock * v;
    float step[3], tmax[3], tdel[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        step[k] = (d[k] > 0) ? 1.0f : -1.0f;
        const float sc = (step[k] > 0) ? 1.0f : 0.0f;
        const float bnd = ((float)c[k] + sc) * ext - 0.5f * v;
        tmax[k] = (bnd - st[k]) / d[k];
        tdel[k] = (step[k] * ext) / d[k];
        if (d[k] == 0.0f) {
            tmax[k] = 1e6f;
            tdel[k] = 1e6f;
        }
    }
#pragma unroll 1
    for (int it = 0; it < kMaxDDA; ++it) {
        if (coord_ok(c[0], c[1], c[2])) {
            const unsigned long long k = pack_key(c[0], c[1], c[2]);
            const int slot = set_insert(set, k);
            if (slot < 0) {
                insert_single(s, k, c[0], c[1], c[2]);
                if (ptag) append_parent(s, k, ptag - 1u);
            } else if (ptag) {
                atomicMax(set_tag + slot, ptag);
            }
        } else {
            atomicAdd(&s.ctr->coord_drops, 1u);
            atomicOr(&s.ctr->flags, (uint32_t)VSG_FLAG_COORD_RANGE);
        }
        if (c[0] == e[0] && c[1] == e[1] && c[2] == e[2]) break;
        if (tmax[0] < tmax[1] && tmax[0] < tmax[2]) {
            tmax[0] += tdel[0];
            c[0] += (int)step[0];
        } else if (tmax[1] < tmax[2]) {
            tmax[1] += tdel[1];
            c[1] += (int)step[1];
        } else {
            tmax[2] += tdel[2];
            c[2] += (int)step[2];
        }
    }
}

// One 16x16 pixel tile (tile_x, tile_y) per CTA of kTile*kTile threads.
// kByNormal: Method 2 rays (the scene's alloc_method == 2), else Method 1;
// separate instantiations keep Method 1's register budget as it was.
template <bool kByNormal>
static __device__ __forceinline__ void alloc_tile(const AllocArgs& a, int tile_x, int tile_y) {
    __shared__ unsigned long long set[kSetCap];
    __shared__ unsigned long long list[kSetCap];
    __shared__ uint32_t set_tag[kSetCap];
    __shared__ int list_n;
    __shared__ uint32_t s_zmin, s_zmax, s_nonfinite, s_valid;
    const int tid = threadIdx.x;
    const SceneDev& s = a.s;
    constexpr bool by_normal = kByNormal;
    for (int i = tid; i < kSetCap; i += blockDim.x) {
        set[i] = kKeyEmpty;
        if (by_normal) set_tag[i] = 0u;
    }
    if (tid == 0) {
        list_n = 0;
        s_zmin = 0xFFFFFFFFu;
        s_zmax = 0u;
        s_nonfinite = 0u;
        s_valid = 0u;
    }
    __syncthreads();
    const int px = tile_x * kTile + (tid & (kTile - 1));
    const int py = tile_y * kTile + (tid / kTile);
    if (px < a.W && py < a.H) {
        const size_t pi = (size_t)py * a.W + px;
        const float p0 = __ldg(a.pm + 3 * pi + 0);
        const float p1 = __ldg(a.pm + 3 * pi + 1);
        const float p2 = __ldg(a.pm + 3 * pi + 2);
        // integration validity (VoxelScene.cu:1040-1046) drives the depth band
        float4 prep = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        if (p0 != 0.0f || p1 != 0.0f || p2 != 0.0f) {
            // depthPos_world and cameraDist, VoxelScene.cu:1052-1062
            float Px, Py, Pz;
            xform(a.pose, p0, p1, p2, Px, Py, Pz);
            const float ex = Px - a.pose.T[3], ey = Py - a.pose.T[7], ez = Pz - a.pose.T[11];
            // .w: the squared-distance threshold of cameraDist (sqrt_threshold)
            prep = make_float4(Px, Py, Pz, sqrt_threshold(sqrtf(ex * ex + ey * ey + ez * ez)));
            atomicAdd(&s_valid, 1u);
            if (isfinite(p0) && isfinite(p1) && isfinite(p2)) {
                atomicMin(&s_zmin, f2ord(p2));
                atomicMax(&s_zmax, f2ord(p2));
            } else {
                s_nonfinite = 1u;
            }
        }
        s.pix_world[pi] = prep;
        s.pix_rgb[pi] = (uint32_t)__ldg(a.rgb + 3 * pi) | ((uint32_t)__ldg(a.rgb + 3 * pi + 1) << 8) |
                        ((uint32_t)__ldg(a.rgb + 3 * pi + 2) << 16);
        const float cx = a.pose.T[3], cy = a.pose.T[7], cz = a.pose.T[11];
        if constexpr (!by_normal) {
            // allocBlocksFromDepthMapMethod1Kernel, VoxelScene.cu:547-633:
            // the camera-space segment p.z -+ truncation
            if (!(p2 <= 1e-6f)) {
                float wx, wy, wz;
                xform(a.pose, p0, p1, p2, wx, wy, wz);
                const float rx = wx - cx, ry = wy - cy, rz = wz - cz;
                const float rl = sqrtf(rx * rx + ry * ry + rz * rz);
                if (!(rl < 1e-6f)) {
                    float st[3], en[3];
                    xform(a.pose, p0, p1, p2 - a.trunc, st[0], st[1], st[2]);
                    xform(a.pose, p0, p1, p2 + a.trunc, en[0], en[1], en[2]);
                    dda_ray(s, set, set_tag, st, en, 0u);
                }
            }
        } else if (p0 != 0.0f || p1 != 0.0f || p2 != 0.0f) {
            // allocBlocksFromDepthMapMethod2Kernel, VoxelScene.cu:797-911
            float n0 = __ldg(a.nm + 3 * pi + 0), n1 = __ldg(a.nm + 3 * pi + 1), n2 = __ldg(a.nm + 3 * pi + 2);
            float nl = sqrtf(n0 * n0 + n1 * n1 + n2 * n2);
            if (!(nl < 0.1f)) {
                n0 /= nl;
                n1 /= nl;
                n2 /= nl;
                float w[3];
                xform(a.pose, p0, p1, p2, w[0], w[1], w[2]);
                const float* T = a.pose.T;
                float nw[3] = {T[0] * n0 + T[1] * n1 + T[2] * n2, T[4] * n0 + T[5] * n1 + T[6] * n2,
                               T[8] * n0 + T[9] * n1 + T[10] * n2};
                nl = sqrtf(nw[0] * nw[0] + nw[1] * nw[1] + nw[2] * nw[2]);
                if (nl > 1e-6f) {
                    nw[0] /= nl;
                    nw[1] /= nl;
                    nw[2] /= nl;
                }
                // camera ray: from the point to truncation behind it
                float rd[3] = {w[0] - cx, w[1] - cy, w[2] - cz};
                const float rl = sqrtf(rd[0] * rd[0] + rd[1] * rd[1] + rd[2] * rd[2]);
                if (rl > 0.0f) {
                    rd[0] /= rl;
                    rd[1] /= rl;
                    rd[2] /= rl;
                    const float en[3] = {w[0] + rd[0] * a.trunc, w[1] + rd[1] * a.trunc, w[2] + rd[2] * a.trunc};
                    dda_ray(s, set, set_tag, w, en, 0u);
                }
                // normal ray: from the point to truncation inside the surface;
                // its blocks take this pixel as parent
                const float en[3] = {w[0] - nw[0] * a.trunc, w[1] - nw[1] * a.trunc, w[2] - nw[2] * a.trunc};
                dda_ray(s, set, set_tag, w, en, (((uint32_t)py << 16) | (uint32_t)px) + 1u);
            }
        }
    }
    __syncthreads();
    for (int i = tid; i < kSetCap; i += blockDim.x) {
        const unsigned long long k = set[i];
        if (k != kKeyEmpty) {
            list[atomicAdd(&list_n, 1)] = k;
            if (by_normal && set_tag[i]) append_parent(s, k, set_tag[i] - 1u);
        }
    }
    __syncthreads();
    const int n = list_n;
    const int warp = tid >> 5, lane = tid & 31;
    const int nwarps = blockDim.x >> 5;
    for (int base = warp * 4; base < n; base += nwarps * 4) {
        const int i = base + (lane >> 3);
        coop_insert(s, i < n ? list[i] : 0ull, i < n);
    }
    if (tid == 0) {
        if (s_valid) {
            atomicAdd(&s.frame->n_valid_px, s_valid);
            if (s_zmin != 0xFFFFFFFFu) {
                atomicMin(&s.frame->zmin_ord, s_zmin);
                atomicMax(&s.frame->zmax_ord, s_zmax);
            }
            if (s_nonfinite) atomicOr(&s.frame->nonfinite, 1u);
        }
    }
}

// After a normal-direction allocation: each (block, pixel) record raises
// the block's parent to (frame + 1) << 32 | y << 16 | x.  Of several normal
// rays through one block in a frame the last pixel in row-major order
// wins (the reference keeps whichever write lands last).
static __device__ __forceinline__ void apply_parents(const SceneDev& s, uint32_t first, uint32_t stride) {
    const uint32_t n = min(*(volatile uint32_t*)&s.frame->n_parent, s.parent_cap);
    const unsigned long long fr = (unsigned long long)(s.frame_seq + 1u) << 32;
    for (uint32_t i = first; i < n; i += stride) {
        const unsigned long long key = s.parent_key[i];
        int x, y, z;
        unpack_key(key, x, y, z);
        const int b = lookup_block(s, key, x, y, z);
        if (b >= 0) atomicMax(s.block_parent + b, fr | (unsigned long long)s.parent_tag[i]);
    }
}

// The parent pixel a block integrates from this frame (VoxelScene.cu:
// 1015-1035): its stored parent when that lies inside this frame's image
// and holds a point; else -1 (each voxel projects).
static __device__ __forceinline__ int parent_pixel(const SceneDev& s, int blk, int W, int H) {
    const unsigned long long t = s.block_parent[blk];
    if (!t) return -1;
    const int x = (int)(t & 0xFFFFu), y = (int)((t >> 16) & 0xFFFFu);
    if (x >= W || y >= H) return -1;
    const int pi = y * W + x;
    return s.pix_world[pi].w < 0.0f ? -1 : pi;
}

// ====================================================================
// integration
// ====================================================================

struct IntegArgs {
    SceneDev s;
    int W, H;
    float trunc;
    Pose pose;
    float fx, fy, cx, cy;
};

// Can any voxel of block (bx,by,bz) be updated this frame?  Conservative:
// a voxel updates only if its rounded projection lands in the image and the
// point it meets is within the truncation distance, so its camera z lies in
// [zmin - t, zmax + t] of the frame's valid points.  Corner projections
// bound the block's projection when it lies in front of the camera.
static __device__ bool block_maybe_updated(const IntegArgs& a, int bx, int by, int bz, float zlo, float zhi) {
    const float v = a.s.voxel;
    const float T3 = a.pose.T[3], T7 = a.pose.T[7], T11 = a.pose.T[11];
    float zmn = 3.4e38f, zmx = -3.4e38f, umn = 3.4e38f, umx = -3.4e38f, vmn = 3.4e38f, vmx = -3.4e38f;
    bool front = zlo > 0.0f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float wx = (float)(bx * 8 + ((c & 1) ? 7 : 0)) * v - T3;
        const float wy = (float)(by * 8 + ((c & 2) ? 7 : 0)) * v - T7;
        const float wz = (float)(bz * 8 + ((c & 4) ? 7 : 0)) * v - T11;
        const float x = a.pose.T[0] * wx + a.pose.T[4] * wy + a.pose.T[8] * wz;
        const float y = a.pose.T[1] * wx + a.pose.T[5] * wy + a.pose.T[9] * wz;
        const float z = a.pose.T[2] * wx + a.pose.T[6] * wy + a.pose.T[10] * wz;
        zmn = fminf(zmn, z);
        zmx = fmaxf(zmx, z);
        if (z > 0.5f * zlo) {
            const float iz = 1.0f / z;
            const float u = x * a.fx * iz + a.cx, w = y * a.fy * iz + a.cy;
            umn = fminf(umn, u);
            umx = fmaxf(umx, u);
            vmn = fminf(vmn, w);
            vmx = fmaxf(vmx, w);
        } else {
            front = false;
        }
    }
    if (zmx < zlo || zmn > zhi) return false;
    if (!front) return true;
    const float m = 2.0f;
    if (umx < -1.5f - m || umn > (float)a.W - 0.5f + m) return false;
    if (vmx < -1.5f - m || vmn > (float)a.H - 0.5f + m) return false;
    return true;
}

// Can a voxel of block (bx,by,bz) lie within the truncation distance of
// the world point P its parent pixel gives every voxel?  Distance from P to
// the box of the block's voxel centres, with a rounding margin.
static __device__ __forceinline__ bool parent_near(const IntegArgs& a, int bx, int by, int bz, float4 P) {
    if (!(isfinite(P.x) && isfinite(P.y) && isfinite(P.z))) return true;
    const float v = a.s.voxel, eps = 1e-3f + 2.0f * v;
    const float p[3] = {P.x, P.y, P.z};
    const int b[3] = {bx, by, bz};
    float d2 = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float lo = (float)(b[k] * 8) * v - eps, hi = (float)(b[k] * 8 + 7) * v + eps;
        const float d = p[k] < lo ? lo - p[k] : (p[k] > hi ? p[k] - hi : 0.0f);
        d2 += d * d;
    }
    const float r = a.trunc + eps;
    return d2 <= r * r;
}

// Visible-block compaction: one thread per pool block in [0, high_water),
// ballot + popc, one atomic per warp.  Stands in for compactifyHashKernel
// (VoxelScene.cu:1275-1300), which lists every allocated block: blocks the
// test rejects cannot have a voxel updated this frame, so integrating only
// the listed ones leaves every voxel as the full pass would.
// Pool blocks first, first + stride, ... of one scene (called by whole CTAs).
static __device__ __forceinline__ void select_blocks(const IntegArgs& a, uint32_t first, uint32_t stride) {
    const SceneDev& s = a.s;
    const int lane = threadIdx.x & 31;
    const uint32_t hw = *(volatile uint32_t*)&s.ctr->high_water;
    const FrameCounters fc = *s.frame;
    const bool any_valid = fc.n_valid_px > 0;
    const bool cull = fc.nonfinite == 0u && fc.zmin_ord != 0xFFFFFFFFu;
    const float eps = 1e-3f + 2.0f * s.voxel;
    const float zlo = cull ? ord2f(fc.zmin_ord) - a.trunc - eps : 0.0f;
    const float zhi = cull ? ord2f(fc.zmax_ord) + a.trunc + eps : 0.0f;
    for (uint32_t b0 = first; b0 < hw; b0 += stride) {
        const uint32_t b = b0 + threadIdx.x;
        bool vis = false;
        if (b < hw) {
            const unsigned long long key = s.block_key[b];
            if (key != kKeyEmpty && key != kKeyTomb) {
                if (s.block_fresh[b]) {
                    vis = true;
                } else if (any_valid) {
                    const int pp = parent_pixel(s, (int)b, a.W, a.H);
                    if (pp >= 0) {
                        int bx, by, bz;
                        unpack_key(key, bx, by, bz);
                        vis = parent_near(a, bx, by, bz, s.pix_world[pp]);
                    } else if (!cull) {
                        vis = true;
                    } else {
                        int bx, by, bz;
                        unpack_key(key, bx, by, bz);
                        vis = block_maybe_updated(a, bx, by, bz, zlo, zhi);
                    }
                }
            }
        }
        const unsigned mask = __ballot_sync(0xFFFFFFFFu, vis);
        if (!mask) continue;
        uint32_t pos = 0;
        if (lane == 0) pos = atomicAdd(&s.frame->n_visible, (uint32_t)__popc(mask));
        pos = __shfl_sync(0xFFFFFFFFu, pos, 0);
        if (vis) s.visible[pos + __popc(mask & ((1u << lane) - 1u))] = b;
    }
}

constexpr int kIntegBatch = 4;  // voxels per lane with loads in flight together

// Per-voxel TSDF update, VoxelScene.cu:954-1126, for the 16 voxels lane
// `lane` owns in block blk (idx = 32k + lane), in batches of kIntegBatch:
// projection of the whole batch, then its point gathers, then the SDF
// decisions, then the voxel / colour loads, then the updates.
static __device__ void integrate_block(const IntegArgs& a, int blk, unsigned long long key, bool fresh, int lane) {
    const SceneDev& s = a.s;
    int bx, by, bz;
    unpack_key(key, bx, by, bz);
    Voxel* vb = s.voxels + (size_t)blk * kVoxPerBlock;
    const float v = s.voxel;
    const float* T = a.pose.T;
    const float camx = T[3], camy = T[7], camz = T[11];
    const float t = a.trunc;
    const int lx = lane & 7;
    const float wx = (float)(int)((unsigned)bx * 8u + (unsigned)lx) * v;
    const float rx = wx - T[3];
    const int ppix = parent_pixel(s, blk, a.W, a.H);
    int cnt = 0;
    unsigned long long wm = 0ull;  // sub-cubes that received a weight this frame
#pragma unroll 1
    for (int k0 = 0; k0 < 16; k0 += kIntegBatch) {
        int pix[kIntegBatch];
#pragma unroll
        for (int j = 0; j < kIntegBatch; ++j) {
            const int k = k0 + j;
            const int ly = (lane >> 3) + ((k & 1) << 2);
            const int lz = k >> 1;
            const float wy = (float)(int)((unsigned)by * 8u + (unsigned)ly) * v;
            const float wz = (float)(int)((unsigned)bz * 8u + (unsigned)lz) * v;
            const float ry = wy - T[7], rz = wz - T[11];
            const float cxp = T[0] * rx + T[4] * ry + T[8] * rz;
            const float cyp = T[1] * rx + T[5] * ry + T[9] * rz;
            const float czp = T[2] * rx + T[6] * ry + T[10] * rz;
            const float sx = cxp * a.fx / czp + a.cx;
            const float sy = cyp * a.fy / czp + a.cy;
            const int ix = __float2int_rz(sx + 0.5f), iy = __float2int_rz(sy + 0.5f);
            pix[j] = ppix >= 0 ? ppix : ((ix >= 0 && ix < a.W && iy >= 0 && iy < a.H) ? iy * a.W + ix : -1);
        }
        float4 P[kIntegBatch];
#pragma unroll
        for (int j = 0; j < kIntegBatch; ++j)
            P[j] = pix[j] >= 0 ? __ldg(s.pix_world + pix[j]) : make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        float sdfv[kIntegBatch];
        bool upd[kIntegBatch];
#pragma unroll
        for (int j = 0; j < kIntegBatch; ++j) {
            const int k = k0 + j;
            const int ly = (lane >> 3) + ((k & 1) << 2);
            const int lz = k >> 1;
            const float wy = (float)(int)((unsigned)by * 8u + (unsigned)ly) * v;
            const float wz = (float)(int)((unsigned)bz * 8u + (unsigned)lz) * v;
            upd[j] = false;
            sdfv[j] = 0.0f;
            if (!(P[j].w < 0.0f)) {  // pixel valid: point != (0,0,0)
                const float dx = wx - P[j].x, dy = wy - P[j].y, dz = wz - P[j].z;
                float sdf = sqrtf(dx * dx + dy * dy + dz * dz);
                // voxelDist < cameraDist, decided on the squared voxel distance
                const float vd2 = (wx - camx) * (wx - camx) + (wy - camy) * (wy - camy) + (wz - camz) * (wz - camz);
                if (vd2 < P[j].w) sdf = -sdf;
                if (!(sdf < -t || sdf > t)) {
                    sdfv[j] = fmaxf(-t, fminf(t, sdf));
                    upd[j] = true;
                }
            }
        }
        Voxel old[kIntegBatch];
        uint32_t col[kIntegBatch];
#pragma unroll
        for (int j = 0; j < kIntegBatch; ++j) {
            const int idx = (k0 + j) * 32 + lane;
            old[j] = Voxel{0.0f, 0u};
            col[j] = 0u;
            if (upd[j]) {
                if (!fresh) old[j] = vb[idx];
                col[j] = __ldg(s.pix_rgb + pix[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < kIntegBatch; ++j) {
            const int idx = (k0 + j) * 32 + lane;
            if (upd[j]) {
                const uint32_t ow = old[j].rgbw >> 24;
                const float oldW = (float)ow;
                const float newW = oldW + 1.0f;
                const float yw = __ldg(s.avg_recip + ow + 1u);  // RN(1 / newW), 0: IEEE division
                const float nsdf = avg_div(old[j].sdf * oldW + sdfv[j] * 1.0f, newW, yw);
                const uint32_t nw = (uint32_t)fminf(255.0f, newW);
                const float nr = avg_div((float)(old[j].rgbw & 0xFFu) * oldW + (float)(col[j] & 0xFFu) * 1.0f, newW, yw);
                const float ng = avg_div(
                    (float)((old[j].rgbw >> 8) & 0xFFu) * oldW + (float)((col[j] >> 8) & 0xFFu) * 1.0f, newW, yw);
                const float nb = avg_div(
                    (float)((old[j].rgbw >> 16) & 0xFFu) * oldW + (float)((col[j] >> 16) & 0xFFu) * 1.0f, newW, yw);
                Voxel nv;
                nv.sdf = nsdf;
                nv.rgbw = pack_rgbw((uint32_t)nr, (uint32_t)ng, (uint32_t)nb, nw);
                vb[idx] = nv;
                ++cnt;
                const int k = k0 + j;
                const int ly = (lane >> 3) + ((k & 1) << 2), lz = k >> 1;
                wm |= 1ull << ((((lz >> 1) * 4 + (ly >> 1)) * 4) + (lx >> 1));
            } else if (fresh) {
                vb[idx] = Voxel{0.0f, 0u};
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, o);
    const unsigned wlo = __reduce_or_sync(0xFFFFFFFFu, (unsigned)wm);
    const unsigned whi = __reduce_or_sync(0xFFFFFFFFu, (unsigned)(wm >> 32));
    const unsigned long long old_wm = fresh ? 0ull : s.block_wmask[blk];
    const unsigned long long newbits = (((unsigned long long)whi << 32) | wlo) & ~old_wm;
    if (newbits && lane < 27) {
        // newly weighted sub-cubes: dilate by one sub-cube into this block
        // position and its 26 neighbours (one lane per neighbour)
        const int dx = lane % 3 - 1, dy = (lane / 3) % 3 - 1, dz = lane / 9 - 1;
        const unsigned long long mk = dil_z(dil_y(dil_x(newbits, dx), dy), dz);
        if (mk) {
            const int nx = bx + dx, ny = by + dy, nz = bz + dz;
            atomicOr(s.dwm + bidx_cell(nx, ny, nz, s.bidx_log2), mk);
            const uint32_t q = grid_bit(nx >> 3, ny >> 3, nz >> 3, s.bidx_log2 - 3);
            atomicOr(s.sup + (q >> 5), 1u << (q & 31));
        }
    }
    __syncwarp();
    if (lane == 0) {
        if (cnt) {
            atomicAdd(&s.frame->n_upd_blocks, 1u);
            atomicAdd(&s.frame->n_upd_voxels, (uint32_t)cnt);
        }
        // only this warp touches the block during the launch
        const unsigned long long nw = ((unsigned long long)whi << 32) | wlo;
        if (fresh) {
            s.block_wmask[blk] = nw;
            s.block_fresh[blk] = 0;
        } else if (nw) {
            s.block_wmask[blk] |= nw;
        }
    }
}

// One warp per visible block, taken from the scene's work counter.
static __device__ __forceinline__ void integrate_work(const IntegArgs& a) {
    const SceneDev& s = a.s;
    const int lane = threadIdx.x & 31;
    const uint32_t n = *(volatile uint32_t*)&s.frame->n_visible;
    for (;;) {
        uint32_t i = 0;
        if (lane == 0) i = atomicAdd(&s.frame->work, 1u);
        i = __shfl_sync(0xFFFFFFFFu, i, 0);
        if (i >= n) break;
        const uint32_t b = s.visible[i];
        const unsigned long long key = s.block_key[b];
        const bool fresh = s.block_fresh[b] != 0;
        integrate_block(a, (int)b, key, fresh, lane);
    }
}

static __device__ __forceinline__ void frame_begin(FrameCounters* f) {
    FrameCounters z = {};
    z.zmin_ord = 0xFFFFFFFFu;
    *f = z;
}

}  // namespace vsg
