/*
 * vsg_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the VoxelSG fusion hot path (block allocation, TSDF
 * integration, ray casting, marching cubes).  It is the parity checker for
 * the CUDA library: only the tests, the smoke check and the CPU-baseline leg
 * of the benchmark load it.  Nothing in the product links or calls it.
 *
 * Every function restates the reference kernel named in its comment
 * (file:line within the VoxelSG project).  Floating point follows the
 * reference operation by operation in IEEE binary32 with no contraction
 * (build with -ffp-contract=off, no fast-math), so integer decisions (pixel
 * rounding, DDA steps, truncation rejects, marching-cubes signs) are
 * reproducible bit for bit.  Float->int conversions emulate the CUDA
 * saturating round-toward-zero conversion (NaN -> 0), which the reference
 * relies on implicitly for pixels that project from behind the camera.
 *
 * Documented semantic choices (the reference behaviour they replace is a
 * scheduling race, not a specification):
 *  - "ideal" allocation: every block the per-pixel DDA visits is allocated.
 *    The reference takes a per-bucket lock at most once per frame and never
 *    releases it (VoxelScene.cu:176-203), so a second new block hashing to
 *    the same bucket in the same frame is dropped at random.
 *  - integration visits every allocated block (VoxelScene.cu:1275-1300 puts
 *    all of them in the compact list); voxels that do not project into a
 *    valid pixel inside the truncation band are left untouched.
 *  - the write-only voxel flags isUpdated / isZeroCrossing are not kept:
 *    nothing on the path reads them.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define BS 8
#define VPB 512
#define KEY_EMPTY 0xFFFFFFFFFFFFFFFFull
#define COORD_LIM (1 << 20)

typedef struct {
    float sdf;
    uint8_t r, g, b, w;
} ovox; /* canonical 8-byte voxel: sdf, colour, weight */

typedef struct {
    float voxel;
    /* open-addressing map: packed block key -> block index */
    uint64_t* mkeys;
    int32_t* mvals;
    int64_t mcap;
    /* dense block storage */
    int64_t n, cap;
    uint64_t* keys;
    ovox* vox;
    /* normal-direction allocation (VoxelScene.cu:768-912): per block the
     * parent pixel of the last normal ray through it, (frame + 1) << 32 |
     * y << 16 | x, 0 = none */
    uint64_t* parent;
    uint32_t frames; /* frames integrated since reset */
    int alloc_method; /* 1 (camera-z band) or 2 (camera + normal rays) */
    int64_t coord_range_drops;
} orc_scene;

/* ---------------------------------------------------------------- helpers */

/* CUDA cvt.rzi.s32.f32: truncation toward zero, saturating, NaN -> 0. */
static inline int32_t f2i(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}

static inline int32_t wrap_sub7(int32_t a) { return (int32_t)((uint32_t)a - 7u); }

static inline uint64_t pack_key(int32_t x, int32_t y, int32_t z) {
    const uint64_t m = 0x1FFFFFull;
    return (((uint64_t)(uint32_t)x & m) << 42) | (((uint64_t)(uint32_t)y & m) << 21) |
           ((uint64_t)(uint32_t)z & m);
}

static inline int32_t sext21(uint64_t v) {
    v &= 0x1FFFFFull;
    return (int32_t)(v & 0x100000ull ? (v | 0xFFFFFFFFFFE00000ull) : v);
}

static inline void unpack_key(uint64_t k, int32_t* b) {
    b[0] = sext21(k >> 42);
    b[1] = sext21(k >> 21);
    b[2] = sext21(k);
}

static inline int in_range(const int32_t* b) {
    return b[0] >= -COORD_LIM && b[0] < COORD_LIM && b[1] >= -COORD_LIM && b[1] < COORD_LIM &&
           b[2] >= -COORD_LIM && b[2] < COORD_LIM;
}

static inline uint64_t mix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

/* Bucket hash of the reference, VoxelScene.cu:61-66 (32-bit wrapping). */
uint32_t orc_bucket_hash(int32_t x, int32_t y, int32_t z, uint32_t num_buckets) {
    uint32_t h = ((uint32_t)x * 73856093u) ^ ((uint32_t)y * 19349663u) ^ ((uint32_t)z * 83492791u);
    return h % num_buckets;
}

/* ---------------------------------------------------------------- CPU map */

static int64_t map_find(const orc_scene* s, uint64_t key) {
    if (s->mcap == 0) return -1;
    uint64_t m = (uint64_t)s->mcap - 1;
    uint64_t i = mix64(key) & m;
    for (;;) {
        uint64_t k = s->mkeys[i];
        if (k == key) return s->mvals[i];
        if (k == KEY_EMPTY) return -1;
        i = (i + 1) & m;
    }
}

static void map_put_raw(uint64_t* mk, int32_t* mv, int64_t cap, uint64_t key, int32_t val) {
    uint64_t m = (uint64_t)cap - 1;
    uint64_t i = mix64(key) & m;
    while (mk[i] != KEY_EMPTY) i = (i + 1) & m;
    mk[i] = key;
    mv[i] = val;
}

static void map_grow(orc_scene* s, int64_t need) {
    if (s->mcap >= 2 * need && s->mcap > 0) return;
    int64_t cap = s->mcap ? s->mcap : 1024;
    while (cap < 2 * need) cap *= 2;
    uint64_t* mk = (uint64_t*)malloc(sizeof(uint64_t) * cap);
    int32_t* mv = (int32_t*)malloc(sizeof(int32_t) * cap);
    for (int64_t i = 0; i < cap; i++) mk[i] = KEY_EMPTY;
    for (int64_t i = 0; i < s->n; i++) map_put_raw(mk, mv, cap, s->keys[i], (int32_t)i);
    free(s->mkeys);
    free(s->mvals);
    s->mkeys = mk;
    s->mvals = mv;
    s->mcap = cap;
}

/* insert a block (zero voxels) if absent; returns 1 when new */
static int scene_add(orc_scene* s, uint64_t key) {
    if (map_find(s, key) >= 0) return 0;
    if (s->n + 1 > s->cap) {
        int64_t nc = s->cap ? s->cap * 2 : 1024;
        s->keys = (uint64_t*)realloc(s->keys, sizeof(uint64_t) * nc);
        s->vox = (ovox*)realloc(s->vox, sizeof(ovox) * VPB * nc);
        s->parent = (uint64_t*)realloc(s->parent, sizeof(uint64_t) * nc);
        s->cap = nc;
    }
    map_grow(s, s->n + 1);
    s->keys[s->n] = key;
    s->parent[s->n] = 0;
    memset(s->vox + s->n * VPB, 0, sizeof(ovox) * VPB);
    map_put_raw(s->mkeys, s->mvals, s->mcap, key, (int32_t)s->n);
    s->n++;
    return 1;
}

orc_scene* orc_create(float voxel) {
    orc_scene* s = (orc_scene*)calloc(1, sizeof(orc_scene));
    s->voxel = voxel;
    s->alloc_method = 1;
    return s;
}

void orc_reset(orc_scene* s) {
    s->n = 0;
    if (s->mkeys)
        for (int64_t i = 0; i < s->mcap; i++) s->mkeys[i] = KEY_EMPTY;
    s->coord_range_drops = 0;
    s->frames = 0;
}

void orc_set_alloc_method(orc_scene* s, int method) { s->alloc_method = method; }

void orc_destroy(orc_scene* s) {
    if (!s) return;
    free(s->mkeys);
    free(s->mvals);
    free(s->keys);
    free(s->vox);
    free(s->parent);
    free(s);
}

int64_t orc_num_blocks(const orc_scene* s) { return s->n; }
int64_t orc_coord_range_drops(const orc_scene* s) { return s->coord_range_drops; }

/* ------------------------------------------------------- allocation (DDA) */

/* worldToSDFBlock, VoxelScene.cu:74-96: voxel = int(p/v + 0.5*sign)
 * (truncation toward zero), negative voxels shifted by -7, then C division. */
static inline void world_to_block_alloc(const float* p, float v, int32_t* b) {
    for (int a = 0; a < 3; a++) {
        float q = p[a] / v;
        float sg = (q > 0) ? 1.0f : ((q < 0) ? -1.0f : 0.0f);
        int32_t iv = f2i(q + sg * 0.5f);
        if (iv < 0) iv = wrap_sub7(iv);
        b[a] = iv / BS;
    }
}

/* row-major camera->world transform of a camera-space point,
 * VoxelScene.cu:561-565 (same operation order everywhere in the reference) */
static inline void xform_point(const float* T, const float* p, float* o) {
    o[0] = T[0] * p[0] + T[1] * p[1] + T[2] * p[2] + T[3];
    o[1] = T[4] * p[0] + T[5] * p[1] + T[6] * p[2] + T[7];
    o[2] = T[8] * p[0] + T[9] * p[1] + T[10] * p[2] + T[11];
}

/* allocateBlocksAlongRay, VoxelScene.cu:295-481.  Writes the visited block
 * coordinates to out (up to 1024 triples); returns how many. */
int orc_dda_blocks(const float* s, const float* e, float v, int32_t* out) {
    int32_t cur[3], end[3];
    world_to_block_alloc(s, v, cur);
    world_to_block_alloc(e, v, end);
    if (cur[0] == end[0] && cur[1] == end[1] && cur[2] == end[2]) return 0; /* :345-348 */
    float d[3] = {e[0] - s[0], e[1] - s[1], e[2] - s[2]};
    float len = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (len < 1e-6f) return 0;
    d[0] /= len;
    d[1] /= len;
    d[2] /= len;
    float step[3], tmax[3], tdel[3];
    const float ext = (float)BS * v;
    for (int a = 0; a < 3; a++) {
        step[a] = (d[a] > 0) ? 1.0f : -1.0f;
        float sc = (step[a] > 0) ? 1.0f : 0.0f;
        float bnd = ((float)cur[a] + sc) * ext - 0.5f * v; /* :373-377 */
        tmax[a] = (bnd - s[a]) / d[a];
        tdel[a] = (step[a] * ext) / d[a];
    }
    for (int a = 0; a < 3; a++)
        if (d[a] == 0.0f) {
            tmax[a] = 1e6f;
            tdel[a] = 1e6f;
        }
    int n = 0;
    for (int it = 0; it < 1024; it++) { /* :417 */
        out[3 * n + 0] = cur[0];
        out[3 * n + 1] = cur[1];
        out[3 * n + 2] = cur[2];
        n++;
        if (cur[0] == end[0] && cur[1] == end[1] && cur[2] == end[2]) break;
        if (tmax[0] < tmax[1] && tmax[0] < tmax[2]) { /* :464-475 */
            tmax[0] += tdel[0];
            cur[0] += (int32_t)step[0];
        } else if (tmax[1] < tmax[2]) {
            tmax[1] += tdel[1];
            cur[1] += (int32_t)step[1];
        } else {
            tmax[2] += tdel[2];
            cur[2] += (int32_t)step[2];
        }
    }
    return n;
}

/* allocBlocksFromDepthMapMethod1Kernel, VoxelScene.cu:487-633, per pixel.
 * Returns the number of blocks written to out. */
static int pixel_alloc_blocks(const float* p, float trunc, const float* T, const float* cam, float v,
                              int32_t* out) {
    if (p[2] <= 1e-6f) return 0; /* :548 (NaN passes, as on the GPU) */
    float w[3];
    xform_point(T, p, w);
    float rd[3] = {w[0] - cam[0], w[1] - cam[1], w[2] - cam[2]};
    float rl = sqrtf(rd[0] * rd[0] + rd[1] * rd[1] + rd[2] * rd[2]);
    if (rl < 1e-6f) return 0;
    float cmin[3] = {p[0], p[1], p[2] - trunc};
    float cmax[3] = {p[0], p[1], p[2] + trunc};
    float rmin[3], rmax[3];
    xform_point(T, cmin, rmin);
    xform_point(T, cmax, rmax);
    return orc_dda_blocks(rmin, rmax, v, out);
}

/* Allocate every block the per-pixel DDA visits ("ideal" allocation).
 * Returns the number of newly allocated blocks. */
int64_t orc_alloc(orc_scene* s, const float* pm, int W, int H, float trunc, const float* T,
                  const float* cam) {
    int64_t npx = (int64_t)W * H;
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    uint64_t** lists = (uint64_t**)calloc(nthr, sizeof(uint64_t*));
    int64_t* lens = (int64_t*)calloc(nthr, sizeof(int64_t));
    int64_t* caps = (int64_t*)calloc(nthr, sizeof(int64_t));
    int64_t drops = 0;
#pragma omp parallel reduction(+ : drops)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        int32_t* buf = (int32_t*)malloc(sizeof(int32_t) * 3 * 1024);
        uint64_t last = KEY_EMPTY;
#pragma omp for schedule(dynamic, 4096)
        for (int64_t i = 0; i < npx; i++) {
            int n = pixel_alloc_blocks(pm + 3 * i, trunc, T, cam, s->voxel, buf);
            for (int j = 0; j < n; j++) {
                if (!in_range(buf + 3 * j)) {
                    drops++;
                    continue;
                }
                uint64_t k = pack_key(buf[3 * j], buf[3 * j + 1], buf[3 * j + 2]);
                if (k == last) continue;
                last = k;
                if (lens[tid] == caps[tid]) {
                    caps[tid] = caps[tid] ? caps[tid] * 2 : 4096;
                    lists[tid] = (uint64_t*)realloc(lists[tid], sizeof(uint64_t) * caps[tid]);
                }
                lists[tid][lens[tid]++] = k;
            }
        }
        free(buf);
    }
    int64_t added = 0;
    for (int t = 0; t < nthr; t++) {
        for (int64_t j = 0; j < lens[t]; j++) added += scene_add(s, lists[t][j]);
        free(lists[t]);
    }
    free(lists);
    free(lens);
    free(caps);
    s->coord_range_drops += drops;
    return added;
}

/* allocBlocksFromDepthMapMethod2Kernel, VoxelScene.cu:797-911, per pixel:
 * the blocks of the camera ray from the point to truncation behind it
 * (out0) and of the normal ray from the point to truncation inside the
 * surface (out1). */
static void pixel_alloc_blocks_m2(const float* p, const float* nc, float trunc, const float* T, const float* cam,
                                  float v, int32_t* out0, int* n0, int32_t* out1, int* n1) {
    *n0 = *n1 = 0;
    if (p[0] == 0.0f && p[1] == 0.0f && p[2] == 0.0f) return; /* :802 */
    float nl = sqrtf(nc[0] * nc[0] + nc[1] * nc[1] + nc[2] * nc[2]);
    if (nl < 0.1f) return; /* :806 */
    const float n[3] = {nc[0] / nl, nc[1] / nl, nc[2] / nl};
    float w[3];
    xform_point(T, p, w);
    float nw[3] = {T[0] * n[0] + T[1] * n[1] + T[2] * n[2], T[4] * n[0] + T[5] * n[1] + T[6] * n[2],
                   T[8] * n[0] + T[9] * n[1] + T[10] * n[2]}; /* :822-827 */
    nl = sqrtf(nw[0] * nw[0] + nw[1] * nw[1] + nw[2] * nw[2]);
    if (nl > 1e-6f) {
        nw[0] /= nl;
        nw[1] /= nl;
        nw[2] /= nl;
    }
    float rd[3] = {w[0] - cam[0], w[1] - cam[1], w[2] - cam[2]}; /* :840-858 */
    const float rl = sqrtf(rd[0] * rd[0] + rd[1] * rd[1] + rd[2] * rd[2]);
    if (rl > 0.0f) {
        rd[0] /= rl;
        rd[1] /= rl;
        rd[2] /= rl;
        const float e[3] = {w[0] + rd[0] * trunc, w[1] + rd[1] * trunc, w[2] + rd[2] * trunc};
        *n0 = orc_dda_blocks(w, e, v, out0);
    }
    const float e1[3] = {w[0] - nw[0] * trunc, w[1] - nw[1] * trunc, w[2] - nw[2] * trunc}; /* :884-889 */
    *n1 = orc_dda_blocks(w, e1, v, out1);
}

/* Normal-direction allocation of every block either ray visits ("ideal"
 * allocation); each block on a normal ray takes the pixel as parent, the
 * last in row-major order when several rays of the frame cross it.
 * Returns the number of newly allocated blocks. */
int64_t orc_alloc_m2(orc_scene* s, const float* pm, const float* nm, int W, int H, float trunc, const float* T,
                     const float* cam) {
    int64_t npx = (int64_t)W * H;
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    uint64_t** lists = (uint64_t**)calloc(nthr, sizeof(uint64_t*));
    uint32_t** tags = (uint32_t**)calloc(nthr, sizeof(uint32_t*));
    int64_t* lens = (int64_t*)calloc(nthr, sizeof(int64_t));
    int64_t* caps = (int64_t*)calloc(nthr, sizeof(int64_t));
    int64_t drops = 0;
#pragma omp parallel reduction(+ : drops)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        int32_t* b0 = (int32_t*)malloc(sizeof(int32_t) * 3 * 1024);
        int32_t* b1 = (int32_t*)malloc(sizeof(int32_t) * 3 * 1024);
#pragma omp for schedule(dynamic, 4096)
        for (int64_t i = 0; i < npx; i++) {
            int n0, n1;
            pixel_alloc_blocks_m2(pm + 3 * i, nm + 3 * i, trunc, T, cam, s->voxel, b0, &n0, b1, &n1);
            const uint32_t ptag = ((uint32_t)(i / W) << 16) | (uint32_t)(i % W);
            for (int r = 0; r < 2; r++) {
                const int n = r ? n1 : n0;
                const int32_t* buf = r ? b1 : b0;
                for (int j = 0; j < n; j++) {
                    if (!in_range(buf + 3 * j)) {
                        drops++;
                        continue;
                    }
                    if (lens[tid] == caps[tid]) {
                        caps[tid] = caps[tid] ? caps[tid] * 2 : 4096;
                        lists[tid] = (uint64_t*)realloc(lists[tid], sizeof(uint64_t) * caps[tid]);
                        tags[tid] = (uint32_t*)realloc(tags[tid], sizeof(uint32_t) * caps[tid]);
                    }
                    lists[tid][lens[tid]] = pack_key(buf[3 * j], buf[3 * j + 1], buf[3 * j + 2]);
                    tags[tid][lens[tid]] = r ? ptag + 1u : 0u;
                    lens[tid]++;
                }
            }
        }
        free(b0);
        free(b1);
    }
    int64_t added = 0;
    const uint64_t fr = (uint64_t)(s->frames + 1u) << 32;
    for (int t = 0; t < nthr; t++) {
        for (int64_t j = 0; j < lens[t]; j++) {
            added += scene_add(s, lists[t][j]);
            if (tags[t][j]) {
                const int64_t at = map_find(s, lists[t][j]);
                const uint64_t tag = fr | (uint64_t)(tags[t][j] - 1u);
                if (tag > s->parent[at]) s->parent[at] = tag;
            }
        }
        free(lists[t]);
        free(tags[t]);
    }
    free(lists);
    free(tags);
    free(lens);
    free(caps);
    s->coord_range_drops += drops;
    return added;
}

/* ---------------------------------------------------------- integration */

/* integrateDepthMapIntoBlocksKernel, VoxelScene.cu:918-1146, for one voxel.
 * Returns 1 when the voxel was updated. */
static inline int integrate_voxel(ovox* vx, int bx, int by, int bz, int idx, const float* pm,
                                  const uint8_t* rgb, int W, int H, float trunc, const float* T,
                                  const float* cam, float v, float fx, float fy, float cx, float cy,
                                  int64_t parent_pi) {
    int lx = idx % BS, ly = (idx / BS) % BS, lz = idx / (BS * BS);
    /* (blockCoord*8 + local) * voxelSize, :959-963 (int arithmetic wraps) */
    float wx = (float)(int32_t)((uint32_t)bx * 8u + (uint32_t)lx) * v;
    float wy = (float)(int32_t)((uint32_t)by * 8u + (uint32_t)ly) * v;
    float wz = (float)(int32_t)((uint32_t)bz * 8u + (uint32_t)lz) * v;
    float rx = wx - T[3], ry = wy - T[7], rz = wz - T[11]; /* :970-974 */
    float px = T[0] * rx + T[4] * ry + T[8] * rz;          /* :976-980 */
    float py = T[1] * rx + T[5] * ry + T[9] * rz;
    float pz = T[2] * rx + T[6] * ry + T[10] * rz;
    float sx = px * fx / pz + cx; /* :984-987 */
    float sy = py * fy / pz + cy;
    int ix = f2i(sx + 0.5f), iy = f2i(sy + 0.5f); /* :990-993 */
    int64_t pi = parent_pi; /* a valid stored parent pixel, :1015-1035 */
    if (pi < 0) {
        if (!(ix >= 0 && ix < W && iy >= 0 && iy < H)) return 0;
        pi = (int64_t)iy * W + ix;
    }
    const float* P = pm + 3 * pi;
    if (!(P[0] != 0.0f || P[1] != 0.0f || P[2] != 0.0f)) return 0; /* :1040-1046 */
    float Pw[3];
    xform_point(T, P, Pw); /* :1052-1056 */
    float dx = wx - Pw[0], dy = wy - Pw[1], dz = wz - Pw[2];
    float sdf = sqrtf(dx * dx + dy * dy + dz * dz);
    float ex = Pw[0] - cam[0], ey = Pw[1] - cam[1], ez = Pw[2] - cam[2];
    float cdist = sqrtf(ex * ex + ey * ey + ez * ez);
    float vdist = sqrtf((wx - cam[0]) * (wx - cam[0]) + (wy - cam[1]) * (wy - cam[1]) +
                        (wz - cam[2]) * (wz - cam[2]));
    if (vdist < cdist) sdf = -sdf; /* :1064-1066 */
    if (sdf < -trunc || sdf > trunc) return 0;
    sdf = fmaxf(-trunc, fminf(trunc, sdf));
    const uint8_t* c = rgb + 3 * pi;
    /* running average with weight increment 1, :1096-1126 */
    float oldS = vx->sdf;
    float oldW = (float)vx->w;
    float newW = oldW + 1.0f;
    if (newW > 0.0f) {
        vx->sdf = (oldS * oldW + sdf * 1.0f) / newW;
        vx->w = (uint8_t)fminf(255.0f, newW);
        float ncr = ((float)vx->r * oldW + (float)c[0] * 1.0f) / newW;
        float ncg = ((float)vx->g * oldW + (float)c[1] * 1.0f) / newW;
        float ncb = ((float)vx->b * oldW + (float)c[2] * 1.0f) / newW;
        vx->r = (uint8_t)ncr;
        vx->g = (uint8_t)ncg;
        vx->b = (uint8_t)ncb;
    }
    return 1;
}

/* Integrate one frame into every allocated block.  out[0] = blocks with at
 * least one updated voxel, out[1] = updated voxels. */
void orc_integrate_blocks(orc_scene* s, const float* pm, const uint8_t* rgb, int W, int H, float trunc,
                          const float* T, const float* cam, float fx, float fy, float cx, float cy,
                          int64_t* out) {
    int64_t nupd = 0, nvox = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : nupd, nvox)
    for (int64_t b = 0; b < s->n; b++) {
        int32_t bc[3];
        unpack_key(s->keys[b], bc);
        ovox* blk = s->vox + b * VPB;
        /* the block's parent pixel when inside this image and holding a
         * point (VoxelScene.cu:1015-1035) */
        int64_t ppi = -1;
        if (s->parent[b]) {
            const int px = (int)(s->parent[b] & 0xFFFFu), py = (int)((s->parent[b] >> 16) & 0xFFFFu);
            if (px < W && py < H) {
                const float* P = pm + 3 * ((int64_t)py * W + px);
                if (P[0] != 0.0f || P[1] != 0.0f || P[2] != 0.0f) ppi = (int64_t)py * W + px;
            }
        }
        int cnt = 0;
        for (int i = 0; i < VPB; i++)
            cnt += integrate_voxel(blk + i, bc[0], bc[1], bc[2], i, pm, rgb, W, H, trunc, T, cam, s->voxel,
                                   fx, fy, cx, cy, ppi);
        nvox += cnt;
        nupd += cnt > 0;
    }
    out[0] = nupd;
    out[1] = nvox;
}

/* VoxelScene::integrateFromScanData, VoxelScene.cpp:404-833: camera position
 * is the translation column of the row-major camera->world matrix
 * (:462-466); allocation, then integration.  out[0]=new blocks,
 * out[1]=updated blocks, out[2]=updated voxels, out[3]=total blocks. */
void orc_integrate_nm(orc_scene* s, const float* pm, const uint8_t* rgb, const float* nm, int W, int H,
                      float trunc, const float* T, float fx, float fy, float cx, float cy, int64_t* out) {
    float cam[3] = {T[3], T[7], T[11]};
    /* without normals the normal-direction allocation is skipped, as in
     * allocBlocksFromDepthMapCUDA (VoxelScene.cu:1693-1715) */
    out[0] = s->alloc_method == 2 ? (nm ? orc_alloc_m2(s, pm, nm, W, H, trunc, T, cam) : 0)
                                  : orc_alloc(s, pm, W, H, trunc, T, cam);
    int64_t r[2];
    orc_integrate_blocks(s, pm, rgb, W, H, trunc, T, cam, fx, fy, cx, cy, r);
    out[1] = r[0];
    out[2] = r[1];
    out[3] = s->n;
    s->frames++;
}

void orc_integrate(orc_scene* s, const float* pm, const uint8_t* rgb, int W, int H, float trunc,
                   const float* T, float fx, float fy, float cx, float cy, int64_t* out) {
    orc_integrate_nm(s, pm, rgb, NULL, W, H, trunc, T, fx, fy, cx, cy, out);
}

/* ------------------------------------------------------------- ray casting */

/* worldToVirtualVoxelPos / virtualVoxelPosToSDFBlock / virtualVoxelPosToLocal,
 * RayCastRender.cu:17-42 (floorf variant, unlike allocation). */
static inline const ovox* get_voxel(const orc_scene* s, const float* p, uint8_t* mark) {
    int32_t vp[3], b[3], l[3];
    for (int a = 0; a < 3; a++) {
        float q = p[a] / s->voxel;
        float sg = (q > 0) ? 1.0f : ((q < 0) ? -1.0f : 0.0f);
        vp[a] = f2i(floorf(q + 0.5f * sg));
        int32_t t = vp[a];
        if (t < 0) t = wrap_sub7(t);
        b[a] = t / BS;
        l[a] = ((vp[a] % BS) + BS) % BS;
    }
    if (!in_range(b)) return NULL;
    int64_t bi = map_find(s, pack_key(b[0], b[1], b[2]));
    if (bi < 0) return NULL;
    if (mark) mark[bi] = 1;
    return s->vox + bi * VPB + (l[0] + l[1] * BS + l[2] * BS * BS);
}

static inline float frac01(float v) { return v - floorf(v); }

/* trilinearInterpolationSimpleFastFast, RayCastRender.cu:127-215 */
static int trilinear(const orc_scene* s, const float* pos, float* dist, uint8_t* color, uint8_t* mark) {
    const float off = s->voxel;
    float pd[3] = {pos[0] - off / 2.0f, pos[1] - off / 2.0f, pos[2] - off / 2.0f};
    float vf[3] = {pd[0] / s->voxel, pd[1] / s->voxel, pd[2] / s->voxel};
    float wt[3] = {frac01(vf[0]), frac01(vf[1]), frac01(vf[2])};
    float d = 0.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f, vws = 0.0f;
    for (int i = 0; i < 8; i++) {
        float q[3] = {pd[0] + ((i & 1) ? off : 0.0f), pd[1] + ((i & 2) ? off : 0.0f),
                      pd[2] + ((i & 4) ? off : 0.0f)};
        const ovox* vx = get_voxel(s, q, mark);
        if (!vx || vx->w == 0) continue;
        float w = ((i & 1) ? wt[0] : (1.0f - wt[0])) * ((i & 2) ? wt[1] : (1.0f - wt[1])) *
                  ((i & 4) ? wt[2] : (1.0f - wt[2]));
        d += w * vx->sdf;
        cr += w * (float)vx->r;
        cg += w * (float)vx->g;
        cb += w * (float)vx->b;
        vws += w;
    }
    if (vws <= 1e-6f) return 0;
    float inv = 1.0f / vws;
    d *= inv;
    cr *= inv;
    cg *= inv;
    cb *= inv;
    *dist = d;
    if (color) {
        color[0] = (uint8_t)cr;
        color[1] = (uint8_t)cg;
        color[2] = (uint8_t)cb;
    }
    return 1;
}

/* findIntersectionBisection, RayCastRender.cu:229-271 (3 regula-falsi steps) */
static int bisection(const orc_scene* s, const float* o, const float* dir, float d0, float r0, float d1,
                     float r1, float* alpha, uint8_t* color, uint8_t* mark) {
    float a = r0, ad = d0, b = r1, bd = d1, c = 0.0f;
    for (int i = 0; i < 3; i++) {
        c = a + (ad / (ad - bd)) * (b - a);
        float cd;
        float sp[3] = {o[0] + c * dir[0], o[1] + c * dir[1], o[2] + c * dir[2]};
        if (!trilinear(s, sp, &cd, color, mark)) return 0;
        if (ad * cd > 0.0f) {
            a = c;
            ad = cd;
        } else {
            b = c;
            bd = cd;
        }
    }
    *alpha = c;
    return 1;
}

#define MINF 1e10f

/* renderKernel + traverseCoarseGridSimpleSampleAll, RayCastRender.cu:407-517,
 * 276-398.  One pixel.  Returns 1 on a hit. steps_out counts samples. */
static int render_pixel(const orc_scene* s, int x, int y, const float* cam, const float* T, float fx,
                        float fy, float cx, float cy, float minD, float maxD, float* depth, float* pos4,
                        float* col4, float* nrm4, int64_t* steps_out, uint8_t* mark, float* bracket) {
    *depth = MINF;
    for (int k = 0; k < 4; k++) pos4[k] = col4[k] = nrm4[k] = MINF;
    float cd[3] = {((float)x - cx) / fx, ((float)y - cy) / fy, 1.0f};
    float cl = sqrtf(cd[0] * cd[0] + cd[1] * cd[1] + cd[2] * cd[2]);
    if (cl > 1e-6f) {
        cd[0] /= cl;
        cd[1] /= cl;
        cd[2] /= cl;
    }
    float wd[3] = {T[0] * cd[0] + T[1] * cd[1] + T[2] * cd[2], T[4] * cd[0] + T[5] * cd[1] + T[6] * cd[2],
                   T[8] * cd[0] + T[9] * cd[1] + T[10] * cd[2]};
    float wl = sqrtf(wd[0] * wd[0] + wd[1] * wd[1] + wd[2] * wd[2]);
    if (wl > 1e-6f) {
        wd[0] /= wl;
        wd[1] /= wl;
        wd[2] /= wl;
    }
    if (minD == 0 || minD == MINF) return 0;
    if (maxD == 0 || maxD == MINF) return 0;
    float lastSdf = 0.0f, lastAlpha = 0.0f;
    unsigned lastW = 0;
    const float d2r = 1.0f / cd[2];
    float rc = d2r * fmaxf(minD, minD);
    float re = d2r * fminf(maxD, maxD);
    int64_t steps = 0;
    while (rc < re) {
        float p[3] = {cam[0] + rc * wd[0], cam[1] + rc * wd[1], cam[2] + rc * wd[2]};
        float dist;
        steps++;
        if (trilinear(s, p, &dist, NULL, mark)) {
            if (lastW > 0 && lastSdf < 0.0f && dist > 0.0f) {
                if (bracket) {
                    bracket[0] = lastAlpha;
                    bracket[1] = rc;
                }
                float alpha = 0.0f;
                uint8_t c2[3] = {0, 0, 0};
                int b = bisection(s, cam, wd, lastSdf, lastAlpha, dist, rc, &alpha, c2, mark);
                float iso[3] = {cam[0] + alpha * wd[0], cam[1] + alpha * wd[1], cam[2] + alpha * wd[2]};
                float th = s->voxel * 3;
                if (b && fabsf(lastSdf - dist) < th) {
                    if (fabsf(dist) < th) {
                        *depth = alpha / d2r;
                        pos4[0] = iso[0];
                        pos4[1] = iso[1];
                        pos4[2] = iso[2];
                        pos4[3] = 1.0f;
                        col4[0] = (float)c2[0] / 255.0f;
                        col4[1] = (float)c2[1] / 255.0f;
                        col4[2] = (float)c2[2] / 255.0f;
                        col4[3] = 1.0f;
                        *steps_out += steps;
                        return 1;
                    }
                }
            }
            lastSdf = dist;
            lastAlpha = rc;
            lastW = 1;
            rc += s->voxel * 0.5f;
        } else {
            lastW = 0;
            rc += s->voxel * 0.5f;
        }
    }
    *steps_out += steps;
    return 0;
}

/* RayCastRender::render, RayCastRender.cpp:123-183 / rayCastRenderCUDA,
 * RayCastRender.cu:526-620.  T is the row-major camera->world matrix; only
 * its rotation is used, the ray origin is cam.  With no allocated block the
 * reference returns before launching (:552-555) and leaves the outputs
 * untouched; so does this.  stats[0]=hits, [1]=misses, [2]=samples. */
void orc_render(const orc_scene* s, int W, int H, const float* cam, const float* T, float fx, float fy,
                float cx, float cy, float minD, float maxD, float* depth, float* pos4, float* col4,
                float* nrm4, int64_t* stats) {
    stats[0] = stats[1] = stats[2] = 0;
    if (s->n == 0) return;
    int64_t hits = 0, miss = 0, steps = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : hits, miss, steps)
    for (int64_t i = 0; i < (int64_t)W * H; i++) {
        int x = (int)(i % W), y = (int)(i / W);
        int h = render_pixel(s, x, y, cam, T, fx, fy, cx, cy, minD, maxD, depth + i, pos4 + 4 * i,
                             col4 + 4 * i, nrm4 + 4 * i, &steps, NULL, NULL);
        hits += h;
        miss += !h;
    }
    stats[0] = hits;
    stats[1] = miss;
    stats[2] = steps;
}

/* Render a sub-rectangle of rows [y0, y1) only (bounded CPU-baseline
 * samples); outputs are full-frame sized. */
void orc_render_rows(const orc_scene* s, int W, int H, int y0, int y1, const float* cam, const float* T,
                     float fx, float fy, float cx, float cy, float minD, float maxD, float* depth,
                     float* pos4, float* col4, float* nrm4, int64_t* stats) {
    stats[0] = stats[1] = stats[2] = 0;
    if (s->n == 0) return;
    if (y0 < 0) y0 = 0;
    if (y1 > H) y1 = H;
    int64_t hits = 0, miss = 0, steps = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : hits, miss, steps)
    for (int64_t i = (int64_t)y0 * W; i < (int64_t)y1 * W; i++) {
        int x = (int)(i % W), y = (int)(i / W);
        int h = render_pixel(s, x, y, cam, T, fx, fy, cx, cy, minD, maxD, depth + i, pos4 + 4 * i,
                             col4 + 4 * i, nrm4 + 4 * i, &steps, NULL, NULL);
        hits += h;
        miss += !h;
    }
    stats[0] = hits;
    stats[1] = miss;
    stats[2] = steps;
}

/* Distinct blocks the reference ray march reads (any tap that resolves to an
 * allocated block), over the whole image.  Used for the algorithmic-byte
 * count of the ray caster; not part of the reference. */
int64_t orc_render_touched_blocks(const orc_scene* s, int W, int H, const float* cam, const float* T,
                                  float fx, float fy, float cx, float cy, float minD, float maxD) {
    if (s->n == 0) return 0;
    uint8_t* mark = (uint8_t*)calloc(s->n, 1);
    int64_t steps = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : steps)
    for (int64_t i = 0; i < (int64_t)W * H; i++) {
        float d, p4[4], c4[4], n4[4];
        render_pixel(s, (int)(i % W), (int)(i / W), cam, T, fx, fy, cx, cy, minD, maxD, &d, p4, c4, n4,
                     &steps, mark, NULL);
    }
    int64_t n = 0;
    for (int64_t b = 0; b < s->n; b++) n += mark[b];
    free(mark);
    return n;
}

/* --------------------------------------------------------- marching cubes */

/* Corner k of a cube at offset ((k ^ k>>1) & 1, k>>1 & 1, k>>2) and edge e
 * from corner MC_EDGE[e][0] to MC_EDGE[e][1]: the numbering of
 * MarchingCubes.cu:264-285 (MC_CORNER_OFFSET_HOST, MC_EDGE_CONNECTION_HOST). */
static const int MC_EDGE[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                   {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

/* vertexInterp, MarchingCubes.cu:313-327 */
static void mc_interp(float iso, const float* p1, const float* p2, float v1, float v2, float* o) {
    const float denom = v2 - v1;
    if (fabsf(denom) < 1e-6f) {
        for (int i = 0; i < 3; i++) o[i] = 0.5f * (p1[i] + p2[i]);
        return;
    }
    float mu = (iso - v1) / denom;
    mu = fminf(fmaxf(mu, 0.0f), 1.0f);
    for (int i = 0; i < 3; i++) o[i] = p1[i] + mu * (p2[i] - p1[i]);
}

/* computeNormal, MarchingCubes.cu:329-350 */
static void mc_normal(const float* v0, const float* v1, const float* v2, float* n) {
    const float a[3] = {v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2]};
    const float b[3] = {v2[0] - v0[0], v2[1] - v0[1], v2[2] - v0[2]};
    n[0] = a[1] * b[2] - a[2] * b[1];
    n[1] = a[2] * b[0] - a[0] * b[2];
    n[2] = a[0] * b[1] - a[1] * b[0];
    const float len = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (len > 1e-6f) {
        const float inv = 1.0f / len;
        n[0] *= inv;
        n[1] *= inv;
        n[2] *= inv;
    } else {
        n[0] = n[1] = n[2] = 0.0f;
    }
}

/* marchingCubesKernel (MarchingCubes.cu:354-467) over every allocated block
 * (the reference's compact list holds all of them, VoxelScene.cu:1275-1300),
 * cubes with local x, y, z < 7 only (:379).  `tab` is a 256 x 16 case table
 * (triangle edge indices, count in entry 15).  Triangles go out in block
 * order, cube order (z, y, x), table order: 9 floats of vertices and 9 of
 * normals (the face normal three times) each, the first max_tris of them
 * written.  Returns the total triangle count, like the reference's counter. */
int64_t orc_marching_cubes(const orc_scene* s, const uint8_t* tab, float iso, float voxel, int64_t max_tris,
                           float* verts, float* norms) {
    int64_t total = 0;
    const float extent = (float)BS * voxel;
    for (int64_t b = 0; b < s->n; b++) {
        int32_t bc[3];
        unpack_key(s->keys[b], bc);
        const float base[3] = {(float)bc[0] * extent, (float)bc[1] * extent, (float)bc[2] * extent};
        const ovox* vb = s->vox + b * VPB;
        for (int lz = 0; lz < BS - 1; lz++)
            for (int ly = 0; ly < BS - 1; ly++)
                for (int lx = 0; lx < BS - 1; lx++) {
                    float val[8], pos[8][3];
                    int ci = 0;
                    for (int k = 0; k < 8; k++) {
                        const int v[3] = {lx + ((k ^ (k >> 1)) & 1), ly + ((k >> 1) & 1), lz + (k >> 2)};
                        val[k] = vb[(v[2] * BS + v[1]) * BS + v[0]].sdf;
                        for (int i = 0; i < 3; i++) pos[k][i] = base[i] + ((float)v[i] + 0.5f) * voxel;
                        if (val[k] < iso) ci |= 1 << k;
                    }
                    if (ci == 0 || ci == 255) continue; /* empty edge mask */
                    float vl[12][3];
                    for (int e = 0; e < 12; e++) {
                        const int c0 = MC_EDGE[e][0], c1 = MC_EDGE[e][1];
                        if (((ci >> c0) & 1) != ((ci >> c1) & 1))
                            mc_interp(iso, pos[c0], pos[c1], val[c0], val[c1], vl[e]);
                    }
                    const uint8_t* row = tab + ci * 16;
                    for (int t = 0; t < row[15]; t++, total++) {
                        if (total >= max_tris) continue;
                        const float* p0 = vl[row[3 * t]];
                        const float* p1 = vl[row[3 * t + 1]];
                        const float* p2 = vl[row[3 * t + 2]];
                        float n[3];
                        mc_normal(p0, p1, p2, n);
                        float* ov = verts + total * 9;
                        float* on = norms + total * 9;
                        for (int i = 0; i < 3; i++) {
                            ov[i] = p0[i];
                            ov[3 + i] = p1[i];
                            ov[6 + i] = p2[i];
                            on[i] = on[3 + i] = on[6 + i] = n[i];
                        }
                    }
                }
    }
    return total;
}

/* ------------------------------------------------ surface-point extraction */

static ovox voxel_at(const orc_scene* s, const float* p) {
    const ovox* v = get_voxel(s, p, NULL);
    ovox e = {0.0f, 0, 0, 0, 0};
    return v ? *v : e;
}

/* computeNormalFromSDF, RayCastRender.cu:629-677 */
static void sdf_normal(const orc_scene* s, const float* p, float* g) {
    const float eps = s->voxel * 0.5f;
    for (int a = 0; a < 3; a++) {
        float q1[3] = {p[0], p[1], p[2]}, q0[3] = {p[0], p[1], p[2]};
        q1[a] = p[a] + eps;
        q0[a] = p[a] - eps;
        const ovox v1 = voxel_at(s, q1), v0 = voxel_at(s, q0);
        g[a] = (v1.w > 0 && v0.w > 0) ? (v1.sdf - v0.sdf) / (2.0f * eps) : 0.0f;
    }
    const float len = sqrtf(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    if (len > 1e-6f) {
        g[0] /= len;
        g[1] /= len;
        g[2] /= len;
    }
}

/* kernelExtractSurfacePoints (RayCastRender.cu:683-868) over every allocated
 * block, voxels in (z, y, x) order: a voxel with weight >= max(1, minW) and
 * SDF in [minSDF, maxSDF] yields the mean of the zero crossings towards its
 * six neighbours (x+, x-, y+, y-, z+, z-; neighbours inside the block by
 * index, outside through getVoxel at centre +- one voxel), or its centre when
 * there is none and |sdf| < 0.001; colour / 255 and the SDF-gradient normal.
 * Writes float4 records in block order, the first max_pts of them; returns
 * the total count. */
int64_t orc_extract_points(const orc_scene* s, float min_sdf, float max_sdf, uint32_t min_w, int64_t max_pts,
                           float* pos, float* col, float* nrm) {
    static const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    const float v = s->voxel;
    int64_t total = 0;
    for (int64_t b = 0; b < s->n; b++) {
        int32_t bc[3];
        unpack_key(s->keys[b], bc);
        const float base[3] = {(float)(bc[0] * BS) * v, (float)(bc[1] * BS) * v, (float)(bc[2] * BS) * v};
        const ovox* vb = s->vox + b * VPB;
        for (int z = 0; z < BS; z++)
            for (int y = 0; y < BS; y++)
                for (int x = 0; x < BS; x++) {
                    const ovox me = vb[x + y * BS + z * BS * BS];
                    if (me.w == 0 || me.w < min_w) continue;
                    if (me.sdf < min_sdf || me.sdf > max_sdf) continue;
                    const int l[3] = {x, y, z};
                    float c[3];
                    for (int a = 0; a < 3; a++) c[a] = base[a] + ((float)l[a] + 0.5f) * v;
                    float acc[3] = {0.0f, 0.0f, 0.0f};
                    int nv = 0;
                    for (int d = 0; d < 6; d++) {
                        const int nl[3] = {x + off[d][0], y + off[d][1], z + off[d][2]};
                        ovox nb;
                        if (nl[0] < 0 || nl[0] >= BS || nl[1] < 0 || nl[1] >= BS || nl[2] < 0 || nl[2] >= BS) {
                            float q[3];
                            for (int a = 0; a < 3; a++) q[a] = c[a] + (float)off[d][a] * v;
                            nb = voxel_at(s, q);
                        } else {
                            nb = vb[nl[0] + nl[1] * BS + nl[2] * BS * BS];
                        }
                        if (nb.w == 0) continue;
                        if ((me.sdf < 0.0f && nb.sdf > 0.0f) || (me.sdf > 0.0f && nb.sdf < 0.0f)) {
                            const float t = me.sdf / (me.sdf - nb.sdf);
                            for (int a = 0; a < 3; a++) acc[a] += c[a] + (float)off[d][a] * v * t;
                            nv++;
                        }
                    }
                    float iso[3];
                    if (nv == 0) {
                        if (!(fabsf(me.sdf) < 0.001f)) continue;
                        iso[0] = c[0];
                        iso[1] = c[1];
                        iso[2] = c[2];
                    } else {
                        for (int a = 0; a < 3; a++) iso[a] = acc[a] / (float)nv;
                    }
                    float g[3];
                    sdf_normal(s, iso, g);
                    if (total < max_pts) {
                        float* P = pos + 4 * total;
                        float* C = col + 4 * total;
                        float* N = nrm + 4 * total;
                        P[0] = iso[0];
                        P[1] = iso[1];
                        P[2] = iso[2];
                        P[3] = 1.0f;
                        C[0] = (float)me.r / 255.0f;
                        C[1] = (float)me.g / 255.0f;
                        C[2] = (float)me.b / 255.0f;
                        C[3] = 1.0f;
                        N[0] = g[0];
                        N[1] = g[1];
                        N[2] = g[2];
                        N[3] = 0.0f;
                    }
                    total++;
                }
    }
    return total;
}

/* -------------------------------------------------------------- streaming */

/* Weighted merge of two partial averages of one voxel (the library's rule
 * for a block streamed in while resident, or stored twice; the reference
 * has none): weights add (cap 255), SDF and colour are weight-averaged,
 * colour truncated to 8 bits. */
static ovox merge_vox(ovox a, ovox b) {
    if (b.w == 0) return a;
    if (a.w == 0) return b;
    const float fa = (float)a.w, fb = (float)b.w, fw = (float)(a.w + b.w);
    ovox o;
    o.sdf = (a.sdf * fa + b.sdf * fb) / fw;
    o.r = (uint8_t)(uint32_t)(((float)a.r * fa + (float)b.r * fb) / fw);
    o.g = (uint8_t)(uint32_t)(((float)a.g * fa + (float)b.g * fb) / fw);
    o.b = (uint8_t)(uint32_t)(((float)a.b * fa + (float)b.b * fb) / fw);
    o.w = (uint8_t)(a.w + b.w > 255 ? 255 : a.w + b.w);
    return o;
}

void orc_merge_voxels(int64_t n, const uint8_t* a, const uint8_t* b, uint8_t* out) {
    for (int64_t i = 0; i < n; i++) {
        ovox x, y;
        memcpy(&x, a + 8 * i, 8);
        memcpy(&y, b + 8 * i, 8);
        const ovox o = merge_vox(x, y);
        memcpy(out + 8 * i, &o, 8);
    }
}

static void rebuild_map(orc_scene* s) {
    for (int64_t i = 0; i < s->mcap; i++) s->mkeys[i] = KEY_EMPTY;
    for (int64_t i = 0; i < s->n; i++) map_put_raw(s->mkeys, s->mvals, s->mcap, s->keys[i], (int32_t)i);
}

/* streamOutFindBlocksKernel_OPTIMIZED + streamOutCopyBlocksKernel
 * (VoxelStreamingManager.cu:36-84, 258-355): every block whose corner
 * (SDFBlockToWorld, :22-28: int coordinate * 8, then times the voxel size)
 * lies at distance >= radius from c leaves the scene; its coordinates and
 * voxels go to the output (scene order).  Returns how many. */
int64_t orc_stream_out(orc_scene* s, const float* c, float radius, int32_t* coords, uint8_t* voxels) {
    int64_t keep = 0, out = 0;
    for (int64_t i = 0; i < s->n; i++) {
        int32_t b[3];
        unpack_key(s->keys[i], b);
        const float dx = (float)(b[0] * BS) * s->voxel - c[0];
        const float dy = (float)(b[1] * BS) * s->voxel - c[1];
        const float dz = (float)(b[2] * BS) * s->voxel - c[2];
        const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
        if (dist >= radius) {
            memcpy(coords + 3 * out, b, sizeof(b));
            memcpy(voxels + out * VPB * 8, s->vox + i * VPB, VPB * 8);
            out++;
        } else {
            if (keep != i) {
                s->keys[keep] = s->keys[i];
                s->parent[keep] = s->parent[i];
                memcpy(s->vox + keep * VPB, s->vox + i * VPB, sizeof(ovox) * VPB);
            }
            keep++;
        }
    }
    s->n = keep;
    if (out) rebuild_map(s);
    return out;
}

/* Stream-in insertion (streamInHashAllocKernel + streamInHashInitKernel,
 * VoxelStreamingManager.cu:443-714): new positions get the stored voxels,
 * resident ones merge them voxel by voxel. */
void orc_stream_in(orc_scene* s, int64_t n, const int32_t* coords, const uint8_t* voxels) {
    for (int64_t i = 0; i < n; i++) {
        const int32_t* b = coords + 3 * i;
        if (!in_range(b)) {
            s->coord_range_drops++;
            continue;
        }
        const uint64_t k = pack_key(b[0], b[1], b[2]);
        const int64_t at = map_find(s, k);
        if (at < 0) {
            scene_add(s, k);
            memcpy(s->vox + (s->n - 1) * VPB, voxels + i * VPB * 8, VPB * 8);
        } else {
            ovox* dst = s->vox + at * VPB;
            for (int v = 0; v < VPB; v++) {
                ovox x;
                memcpy(&x, voxels + (i * VPB + v) * 8, 8);
                dst[v] = merge_vox(dst[v], x);
            }
        }
    }
}

/* March bracket [lastAlpha, rc] of each hit pixel's zero crossing (float2
 * per pixel; misses untouched): the discrete decision the ray-cast adjoint
 * holds fixed.  Test support, not part of the reference. */
void orc_render_brackets(const orc_scene* s, int W, int H, const float* cam, const float* T, float fx, float fy,
                         float cx, float cy, float minD, float maxD, float* bracket) {
    if (s->n == 0) return;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)W * H; i++) {
        float d, p4[4], c4[4], n4[4], br[2];
        int64_t steps = 0;
        if (render_pixel(s, (int)(i % W), (int)(i / W), cam, T, fx, fy, cx, cy, minD, maxD, &d, p4, c4, n4, &steps,
                         NULL, br)) {
            bracket[2 * i] = br[0];
            bracket[2 * i + 1] = br[1];
        }
    }
}

/* ------------------------------------------------------ point-cloud splat */

/* CustomDepthMapGenerator::generateFromPointCloud (CustomDepthMapGenerator.
 * cpp:81-222): sequential loop over the points (mode 0: every accepted point
 * overwrites its pixel, its normal / colour only when it has one); mode 1
 * keeps the nearest point (the later one on equal z) with its own normal and
 * colour.  Normals from the depth map when n_nrm == 0 (:163-209).  Outputs
 * are zero-initialised here; any may be NULL except depth. */
void orc_splat_points(const float* pts, int64_t n, const float* nrm, int64_t n_nrm, const uint8_t* col,
                      int64_t n_col, int W, int H, float fx, float fy, float cx, float cy, float zmin, float zmax,
                      int mode, float* depth, float* pm, float* nm, uint8_t* cm) {
    const int64_t npx = (int64_t)W * H;
    int64_t* win = (int64_t*)malloc(sizeof(int64_t) * (npx ? npx : 1));
    for (int64_t p = 0; p < npx; p++) win[p] = -1;
    memset(depth, 0, sizeof(float) * npx);
    if (pm) memset(pm, 0, sizeof(float) * 3 * npx);
    if (nm) memset(nm, 0, sizeof(float) * 3 * npx);
    if (cm) memset(cm, 0, 3 * npx);
    for (int64_t i = 0; i < n; i++) {
        const float x = pts[3 * i], y = pts[3 * i + 1], z = pts[3 * i + 2];
        if (z <= 0.0f) continue; /* :114 */
        if (z < zmin || z > zmax) continue;
        const float u = (x * fx / z) + cx; /* :553-556 */
        const float v = (y * fy / z) + cy;
        if (!(u >= 0.0f && u < (float)W && v >= 0.0f && v < (float)H)) continue; /* :586-587 */
        const int px = (int)floorf(u), py = (int)floorf(v);
        if (px < 0 || py < 0 || px >= W || py >= H) continue; /* :142 */
        const int64_t p = (int64_t)py * W + px;
        if (mode == 1 && win[p] >= 0 && pts[3 * win[p] + 2] < z) continue;
        win[p] = i;
        depth[p] = z;
        if (pm) {
            pm[3 * p] = x;
            pm[3 * p + 1] = y;
            pm[3 * p + 2] = z;
        }
        if (nm) {
            if (i < n_nrm) memcpy(nm + 3 * p, nrm + 3 * i, 12);
            else if (mode == 1) memset(nm + 3 * p, 0, 12);
        }
        if (cm) {
            if (i < n_col) memcpy(cm + 3 * p, col + 3 * i, 3);
            else if (mode == 1) memset(cm + 3 * p, 0, 3);
        }
    }
    if (nm && n_nrm == 0) {
        for (int y = 1; y < H - 1; y++)
            for (int x = 1; x < W - 1; x++) {
                const int64_t i = (int64_t)y * W + x;
                const float d = depth[i];
                if (!(d > 0.0f)) continue;
                const float dr = depth[i + 1], dd = depth[i + W];
                const float c[3] = {((float)x - cx) * d / fx, ((float)y - cy) * d / fy, d};
                const float r[3] = {((float)(x + 1) - cx) * dr / fx, ((float)y - cy) * dr / fy, dr};
                const float w[3] = {((float)x - cx) * dd / fx, ((float)(y + 1) - cy) * dd / fy, dd};
                const float a0 = r[0] - c[0], a1 = r[1] - c[1], a2 = r[2] - c[2];
                const float b0 = w[0] - c[0], b1 = w[1] - c[1], b2 = w[2] - c[2];
                const float n0 = a1 * b2 - a2 * b1, n1 = a2 * b0 - a0 * b2, n2 = a0 * b1 - a1 * b0;
                const float len = sqrtf(n0 * n0 + n1 * n1 + n2 * n2);
                if (len > 0.0f) {
                    const float inv = 1.0f / len;
                    nm[3 * i] = n0 * inv;
                    nm[3 * i + 1] = n1 * inv;
                    nm[3 * i + 2] = n2 * inv;
                }
            }
    }
    free(win);
}

/* ------------------------------------------------------- export / import */

static int cmp_key3(const void* a, const void* b) {
    const int32_t* x = (const int32_t*)a;
    const int32_t* y = (const int32_t*)b;
    for (int i = 0; i < 3; i++) {
        if (x[i] < y[i]) return -1;
        if (x[i] > y[i]) return 1;
    }
    return 0;
}

typedef struct {
    int32_t c[3];
    int32_t idx;
} keyidx;

/* Sorted (x, y, z) block coordinates and their 512 voxels each (8 bytes per
 * voxel: sdf f32, r, g, b, weight). */
void orc_export(const orc_scene* s, int32_t* coords, uint8_t* voxels) {
    keyidx* t = (keyidx*)malloc(sizeof(keyidx) * (s->n ? s->n : 1));
    for (int64_t i = 0; i < s->n; i++) {
        unpack_key(s->keys[i], t[i].c);
        t[i].idx = (int32_t)i;
    }
    qsort(t, s->n, sizeof(keyidx), cmp_key3);
    for (int64_t i = 0; i < s->n; i++) {
        memcpy(coords + 3 * i, t[i].c, sizeof(int32_t) * 3);
        if (voxels) memcpy(voxels + i * VPB * 8, s->vox + (int64_t)t[i].idx * VPB, VPB * 8);
    }
    free(t);
}

/* Parent tags of the blocks in orc_export's order (0 = none, else
 * (frame + 1) << 32 | y << 16 | x). */
void orc_export_parents(const orc_scene* s, uint64_t* out) {
    keyidx* t = (keyidx*)malloc(sizeof(keyidx) * (s->n ? s->n : 1));
    for (int64_t i = 0; i < s->n; i++) {
        unpack_key(s->keys[i], t[i].c);
        t[i].idx = (int32_t)i;
    }
    qsort(t, s->n, sizeof(keyidx), cmp_key3);
    for (int64_t i = 0; i < s->n; i++) out[i] = s->parent[t[i].idx];
    free(t);
}

/* Replace the scene with the given blocks (coordinates + 8-byte voxels). */
void orc_import(orc_scene* s, int64_t n, const int32_t* coords, const uint8_t* voxels) {
    orc_reset(s);
    for (int64_t i = 0; i < n; i++) {
        uint64_t k = pack_key(coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]);
        if (scene_add(s, k)) memcpy(s->vox + (s->n - 1) * VPB, voxels + i * VPB * 8, VPB * 8);
    }
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
