/*
 * vsg.h -- C ABI of the B200 fusion library (libvsg.so).
 *
 * Plain C: opaque handles, POD structs, raw pointers and sizes.  Device
 * buffers are CUDA device pointers; streams are cudaStream_t passed as
 * void* (NULL = legacy default stream).  Every entry point returns a status
 * code (VSG_OK = 0) instead of printing and returning void as the reference
 * launchers do.
 *
 * Each entry point replaces a reference interface (paths within the VoxelSG
 * project):
 *   vsg_scene_create / destroy  VoxelScene::VoxelScene / ~VoxelScene,
 *                               CUDAHashRef::HashDataAllocation
 *                               (VoxelScene.h:58-63, CUDAHashRef.cu:40-178)
 *   vsg_scene_reset             VoxelScene::reset, resetHashDataCUDA
 *                               (VoxelScene.h:68, VoxelScene.cu:1166-1236)
 *   vsg_integrate               VoxelScene::integrateFromScanData
 *                               (VoxelScene.h:89-91, VoxelScene.cpp:404-833):
 *                               allocBlocksFromDepthMapCUDA +
 *                               compactifyHashCUDA +
 *                               integrateDepthMapIntoBlocksCUDA
 *                               (VoxelScene.h:22-40)
 *   vsg_renderer_create         RayCastRender::initialize (RayCastRender.h:56)
 *   vsg_render                  RayCastRender::render / rayCastRenderCUDA
 *                               (RayCastRender.h:66-70, RayCastRender.cpp:28-32)
 *   vsg_renderer_outputs        RayCastRender::getOutputDepth/Color/Normal/
 *                               Positions (RayCastRender.h:114-117)
 *   vsg_renderer_download       RayCastRender::downloadResults /
 *                               downloadDepthFloat (RayCastRender.h:78-83)
 *   vsg_scene_stats             VoxelScene::getHeapFreeCount /
 *                               getNumIntegratedFrames / printStats
 *                               (VoxelScene.h:104-115, 177)
 *   vsg_scene_export            VoxelScene::getHashData (VoxelScene.h:129)
 *                               read back to the host as sorted block records
 */
#ifndef VSG_H
#define VSG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define VSG_API __attribute__((visibility("default")))
#else
#define VSG_API
#endif

typedef void* vsg_stream_t; /* cudaStream_t */
typedef struct vsg_scene vsg_scene;
typedef struct vsg_renderer vsg_renderer;

/* status codes */
enum {
    VSG_OK = 0,
    VSG_ERR_INVALID_ARG = 1,   /* null pointer, non-positive size, bad knob */
    VSG_ERR_NOT_ALLOCATED = 2, /* handle not initialised */
    VSG_ERR_CUDA = 3,          /* a CUDA runtime call failed */
    VSG_ERR_OUT_OF_MEMORY = 4, /* device or host allocation failed */
    VSG_ERR_TOO_LARGE = 5      /* a size exceeds a documented maximum */
};

/* sticky device-side condition flags (vsg_stats.flags) */
enum {
    VSG_FLAG_HEAP_EXHAUSTED = 1u,   /* voxel pool ran out; blocks were not allocated */
    VSG_FLAG_CHAIN_EXHAUSTED = 2u,  /* bucket overflow chain pool ran out */
    VSG_FLAG_COORD_RANGE = 4u,      /* a block coordinate outside +-2^20 was skipped */
    VSG_FLAG_INSERT_RETRY = 8u,     /* a bounded insert retry loop gave up */
    VSG_FLAG_MARCH_LIMIT = 16u,     /* a ray hit the iteration guard */
    VSG_FLAG_PARENT_OVERFLOW = 32u  /* normal-direction allocation: a frame's parent records
                                       overflowed (a DDA ran to its 1024-block guard); some
                                       blocks kept an older parent pixel */
};

/* GlobalParamsConfig knobs (globalPramasConfig.h:101-109) and the sizes
 * Params derives from them (CUDAHashData.h:14-29). */
typedef struct vsg_params {
    float voxel_size;         /* g_SDFVoxelSize (m) */
    float truncation;         /* g_SDFTruncation (m); frames pass their own */
    float truncation_scale;   /* g_SDFTruncationScale (not read on the path) */
    uint32_t hash_num_slots;  /* g_hashNumSlots: number of hash buckets */
    uint32_t num_sdf_blocks;  /* g_hashNumSDFBlocks: 8^3-voxel blocks in the pool */
    uint32_t max_chain_nodes; /* bucket-overflow entries; 0 = 2 * hash_num_slots */
    uint32_t occupancy_log2;  /* toroidal block grids (dense index, skip masks) are
                                 2^k block positions per axis, k in 5..9 (0 = 7) */
} vsg_params;

typedef struct vsg_stats {
    uint32_t allocated_blocks;   /* blocks currently in the hash */
    uint32_t free_blocks;        /* heap free count (getHeapFreeCount) */
    uint32_t high_water;         /* highest pool index in use + 1 */
    uint32_t chain_nodes_used;   /* bucket-overflow entries consumed */
    uint32_t integrated_frames;  /* getNumIntegratedFrames */
    uint32_t frame_valid_pixels; /* last frame: pixels with a non-zero point */
    uint32_t frame_new_blocks;   /* last frame: blocks allocated */
    uint32_t frame_visible_blocks; /* last frame: blocks passed to integration */
    uint32_t frame_updated_blocks; /* last frame: blocks with >= 1 voxel updated */
    uint32_t frame_updated_voxels; /* last frame: voxels updated */
    uint32_t render_hits;        /* last render: rays that found a surface */
    uint32_t render_misses;      /* last render: rays that did not */
    uint32_t render_samples_full;    /* last render: march samples evaluated */
    uint32_t render_samples_skipped; /* last render with march statistics on: samples skipped as empty */
    uint32_t render_jumps;           /* last render: O(1) jumps over skipped runs */
    uint32_t render_singles;         /* last render with march statistics on: samples evaluated at a
                                        skip-cell boundary */
    uint32_t render_blocks_read;     /* last render with march statistics on: distinct blocks read */
    uint32_t render_lane_iters;      /* last render: march iterations summed over rays */
    uint32_t render_warp_iters;      /* last render: per-warp maximum iterations, summed */
    uint32_t flags;              /* VSG_FLAG_* (sticky since reset) */
    uint32_t fast_division;      /* 1: the ray caster divides by the voxel size with a
                                    product + correction verified exhaustively against
                                    IEEE division at scene creation */
    uint32_t fast_avg_divisors;  /* of the running average's 256 divisors (new weight
                                    1..256), those whose one-correction product was
                                    verified equal to IEEE division for every dividend */
    uint32_t pixel_buffer_capacity; /* pixels the scene's own per-pixel work buffers hold
                                       (grown by vsg_integrate; 0 if only
                                       vsg_integrate_noalloc has run) */
} vsg_stats;

/* Reference defaults of the knobs used by the tests (README.md:79-83). */
VSG_API int vsg_params_default(vsg_params* p);

VSG_API int vsg_scene_create(const vsg_params* p, vsg_scene** out);
VSG_API int vsg_scene_destroy(vsg_scene* s);
VSG_API int vsg_scene_reset(vsg_scene* s, vsg_stream_t stream);
VSG_API int vsg_scene_params(const vsg_scene* s, vsg_params* out);

/* Integrate one frame: allocate the blocks along each pixel's truncation
 * band, select the blocks the frame can touch, update their voxels.
 * pointmap: device float3[w*h] camera-space points ((0,0,0) = invalid);
 * rgb: device uchar3[w*h]; normals: device float3[w*h] (must be non-null,
 * as in the reference; read only by the normal-direction allocation);
 * pose: HOST float[16] row-major camera->world.  Stream-ordered; does not
 * synchronise. */
VSG_API int vsg_integrate(vsg_scene* s, const float* pointmap, const uint8_t* rgb, const float* normals, int w,
                  int h, float truncation, const float pose[16], float fx, float fy, float cx, float cy,
                  vsg_stream_t stream);

/* Same integration as vsg_integrate, allocating no device memory.  This entry
 * point has no counterpart in the reference.  It is for callers that cannot
 * allocate while integrating: real-time loops that must not stall on
 * cudaMalloc/cudaFree (both can synchronise the whole device), hosts that
 * hand the library a fixed GPU memory budget at start-up, and plug-in hosts
 * whose own allocator owns all device memory.  vsg_integrate grows two per-pixel work buffers with cudaMalloc
 * when it first sees a larger image; this variant takes them from a fixed
 * 20 MiB array of device memory inside the library instead.
 * Limits and rules:
 *   - at most 1,048,576 pixels (w*h) per frame; larger frames return
 *     VSG_ERR_TOO_LARGE without doing anything;
 *   - the first call on each device looks the array's address up
 *     (cudaGetSymbolAddress) and should come before any stream capture; the
 *     address is cached with the id of the device's current context and
 *     looked up again, by the next call, when that context has changed
 *     (after cudaDeviceReset, or with another driver context made current),
 *     so that call too should come before any stream capture;
 *   - its launches are not timed: the vsg_timing_* slots see only
 *     vsg_integrate's frames;
 *   - every call on a device shares the one array, so calls whose work
 *     overlaps on the GPU (other streams, other scenes) race; serialise them;
 *   - the scene must live on the current device (else VSG_ERR_INVALID_ARG);
 *   - scenes set to the normal-direction allocation (method 2) are refused
 *     with VSG_ERR_INVALID_ARG: that allocation keeps per-frame records in
 *     buffers of the scene's own.
 * The scene itself is created beforehand with vsg_scene_create. */
VSG_API int vsg_integrate_noalloc(vsg_scene* s, const float* pointmap, const uint8_t* rgb, const float* normals,
                                  int w, int h, float truncation, const float pose[16], float fx, float fy,
                                  float cx, float cy, vsg_stream_t stream);

/* Allocation mode of vsg_integrate (allocBlocksFromDepthMapCUDA,
 * VoxelScene.cu:1676-1721, chooses at compile time with
 * USE_NORMAL_DIR_ALLOC):
 *   1  (default) Method 1, VoxelScene.cu:487-633: per pixel the blocks of
 *      the camera-space segment p.z -+ truncation;
 *   2  Method 2, VoxelScene.cu:768-912: per pixel with a normal of length
 *      >= 0.1, the blocks of the camera ray from the point to truncation
 *      behind it and of the normal ray from the point to truncation inside
 *      the surface.  A block on a normal ray records the pixel as its
 *      parent (the last such pixel of the last such frame; of one frame's
 *      rays the last in row-major order); integration then updates every
 *      voxel of that block from the parent pixel's point instead of the
 *      voxel's own projection whenever that pixel lies inside the frame and
 *      holds a point (VoxelScene.cu:1015-1035).  Images up to 65535 pixels
 *      on a side (VSG_ERR_TOO_LARGE beyond); not available to
 *      vsg_integrate_noalloc or vsg_batch_step (VSG_ERR_INVALID_ARG).
 * Parents persist until the scene is reset or the block is freed, and are
 * honoured in either mode.  Takes effect at the next vsg_integrate. */
VSG_API int vsg_scene_set_alloc_method(vsg_scene* s, int method);

/* Depth image -> camera-space point map (no counterpart on the reference's
 * path, which receives point maps from CustomDepthMapGenerator,
 * CustomDepthMapGenerator.cpp:81-222): p = ((x - cx) d / fx, (y - cy) d / fy,
 * d) per pixel, (0,0,0) where d is not a positive finite number; normals (may
 * be NULL) as that generator's fallback computes them (:163-209): normalised
 * cross product of the right and lower neighbours' offsets, interior pixels
 * with d > 0, else (0,0,0).  depth: device float[w*h]; pointmap, normals:
 * device float3[w*h].  Stream-ordered. */
/* Point cloud -> depth / point / normal / colour maps on the GPU
 * (CustomDepthMapGenerator::generateFromPointCloud,
 * CustomDepthMapGenerator.cpp:81-222, perspective projection :550-556).
 * A point with z > 0 and min_depth <= z <= max_depth projects to
 * u = x fx / z + cx, v = y fy / z + cy; inside [0, w) x [0, h) it lands on
 * pixel (floor u, floor v).  mode VSG_SPLAT_LAST: the reference's order --
 * the last point in input order wins the pixel, whose normal and colour are
 * those of the last point landing there that has one (index < n_normals,
 * index < n_colors); VSG_SPLAT_NEAREST: the nearest point wins (the later
 * one on equal z) with its own normal and colour (zeros when it has none),
 * the z-buffer of CUDADepthMapData.cu:9-53 without its race.  Pixels
 * without a point hold 0.  With n_normals == 0 the normal map is the
 * generator's fallback over the depth map (:163-209).  Pass min_depth 0 and
 * max_depth INFINITY for the reference's generator, which has no range.
 * points, normals: device float3; colors: device uchar3; outputs (device,
 * each may be NULL): depth float[w*h], pointmap and normalmap float3[w*h],
 * colormap uchar3[w*h].  n_points < 2^32 - 1 (else VSG_ERR_TOO_LARGE).
 * *n_valid (host, may be NULL) receives the pixels that got a point and
 * then the call synchronises; otherwise stream-ordered.  A work buffer of
 * 20 bytes per pixel comes from the stream-ordered allocator. */
enum { VSG_SPLAT_LAST = 0, VSG_SPLAT_NEAREST = 1 };
VSG_API int vsg_splat_points(const float* points, int64_t n_points, const float* normals, int64_t n_normals,
                             const uint8_t* colors, int64_t n_colors, int w, int h, float fx, float fy, float cx,
                             float cy, float min_depth, float max_depth, int mode, float* depth, float* pointmap,
                             float* normalmap, uint8_t* colormap, int64_t* n_valid, vsg_stream_t stream);

VSG_API int vsg_depth_to_pointmap(const float* depth, int w, int h, float fx, float fy, float cx, float cy,
                                  float* pointmap, float* normals, vsg_stream_t stream);

/* Counters of the scene and of its last frame / render.  Synchronises. */
VSG_API int vsg_scene_stats(vsg_scene* s, vsg_stats* out);

/* Read every allocated block back: coords int32[n*3] sorted by (x,y,z) and
 * 512 voxels each as 8-byte records (float sdf, uint8 r, g, b, weight).
 * voxels may be NULL.  Fails with VSG_ERR_TOO_LARGE when more than
 * max_blocks are allocated (n_out still receives the count).  Synchronises. */
VSG_API int vsg_scene_export(vsg_scene* s, int32_t* coords, uint8_t* voxels, uint32_t max_blocks,
                     uint32_t* n_out);

VSG_API int vsg_renderer_create(int w, int h, vsg_renderer** out);
VSG_API int vsg_renderer_destroy(vsg_renderer* r);

/* Ray cast the scene.  pose_dev: DEVICE float[16] row-major camera->world
 * (the reference passes a caller-owned device matrix); only its rotation is
 * read, cam_pos (host float[3]) is the ray origin.  When the scene holds no
 * block the outputs are left untouched, as in the reference.  Two launches
 * on the stream: per-tile march distance bounds (into the renderer's own
 * buffer), then the ray cast; calls on one renderer must not overlap on the
 * GPU (they share its outputs and that buffer). */
VSG_API int vsg_render(vsg_renderer* r, const vsg_scene* s, const float cam_pos[3], const float* pose_dev,
               float fx, float fy, float cx, float cy, float min_depth, float max_depth,
               vsg_stream_t stream);
/* Same with a HOST pose. */
VSG_API int vsg_render_hostpose(vsg_renderer* r, const vsg_scene* s, const float cam_pos[3], const float pose[16],
                        float fx, float fy, float cx, float cy, float min_depth, float max_depth,
                        vsg_stream_t stream);

/* Device output buffers: depth float[w*h]; position, colour, normal float4
 * [w*h].  Misses hold 1e10 in every component. */
VSG_API int vsg_renderer_outputs(const vsg_renderer* r, float** depth, float** position, float** color,
                         float** normal);
/* Copy the outputs to host memory (any pointer may be NULL); synchronous. */
VSG_API int vsg_renderer_download(const vsg_renderer* r, float* depth, float* position, float* color,
                          float* normal);
/* RayCastRender::savePointCloudPLY (RayCastRender.cpp:221-302): ASCII PLY
 * of the last render's hit positions (depth finite, > 0 and < 1e9; position
 * finite) with colour channels clamped to [0, 1] and rounded to 0..255
 * (non-finite -> 255); parent directories are created.  No file and
 * VSG_ERR_INVALID_ARG when no pixel is valid or the file cannot be
 * written.  *n_points (may be NULL) receives the number written.
 * Synchronous. */
VSG_API int vsg_renderer_save_ply(const vsg_renderer* r, const char* path, int64_t* n_points);

/* ---- adjoint of the ray cast (no counterpart in the reference) ----------
 * A hit pixel's depth and position are smooth functions of the camera pose
 * and of the voxel SDF values once the march's discrete decisions are fixed
 * (the zero-crossing bracket, each sample's tap voxels and their weights, the
 * side each regula-falsi step keeps).  vsg_renderer_record makes the
 * following renders keep each pixel's bracket (8 bytes per pixel, allocated
 * on the first enable); vsg_render_backward then recomputes the crossing
 * with the forward's exact arithmetic and runs reverse mode through it.
 * The render must have used the same scene, unchanged since, and the pose's
 * translation as ray origin (vsg_render_hostpose does). */
VSG_API int vsg_renderer_record(vsg_renderer* r, int enable);
/* March step of this renderer's ray casts, in metres (no reference
 * counterpart; the reference always steps half a voxel, RayCastRender.cu:
 * 389-392).  0 (the default) keeps the reference's step and its depths bit
 * for bit.  Any positive value is an opt-in approximation for callers that
 * trade depth accuracy for speed: samples are taken every `step` metres and
 * the crossing is refined as before, so depths move by up to a few
 * millimetres and thin structures can be missed.  Applies to vsg_render,
 * vsg_render_hostpose and the batched step.  Negative or non-finite values:
 * VSG_ERR_INVALID_ARG. */
VSG_API int vsg_renderer_set_step(vsg_renderer* r, float step);
/* grad_depth: device float[w*h] dL/d depth (NULL = 0); grad_position: device
 * float4[w*h] dL/d position (NULL = 0).  grad_pose: DEVICE double[12]
 * receiving dL/dT for the row-major 3x4 camera->world matrix (written;
 * rotation entries 0-2, 4-6, 8-10, translation 3, 7, 11).  grad_sdf: device
 * float[num_sdf_blocks * 512] indexed like the voxel pool (pool block * 512 +
 * x + 8y + 64z), ACCUMULATED with atomics (NULL = skip).  min_weight_sum:
 * leave out pixels where a sample of the crossing renormalises over valid
 * taps whose trilinear weights sum to less (0 keeps every pixel; near the
 * edge of observed space that sum is small and the depth -- hence its
 * gradient -- is steep: 0.5 suits pose optimisation).  n_skipped: if not
 * NULL, the call synchronises and stores the number of hit pixels left out:
 * those whose recomputation did not reproduce the rendered depth (none when
 * the preconditions hold), those below min_weight_sum, and those where the
 * depth has no derivative (a regula-falsi step between two equal values,
 * e.g. samples that read only truncation-clamped voxels, where the forward
 * step is decided by rounding). */
VSG_API int vsg_render_backward(const vsg_renderer* r, const vsg_scene* s, const float pose[16], float fx, float fy,
                                float cx, float cy, const float* grad_depth, const float* grad_position,
                                double* grad_pose, float* grad_sdf, float min_weight_sum, uint32_t* n_skipped,
                                vsg_stream_t stream);
/* Adjoint of one frame's integration (no reference counterpart): call right
 * after the vsg_integrate of that frame, with the same point map, pose,
 * intrinsics and truncation.  grad_sdf: device float[num_sdf_blocks * 512]
 * holding dL/d(voxel SDF after the frame), pool-indexed; for every voxel the
 * frame updated it is replaced IN PLACE by dL/d(SDF before the frame) (the
 * others are unchanged).  grad_pose: DEVICE double[12] receiving dL/dT of the
 * row-major 3x4 camera->world matrix (written); grad_pointmap: device
 * float3[w*h] dL/dp, ACCUMULATED (NULL = skip).  Decisions (each voxel's
 * pixel, sign, truncation test) are the forward's; a voxel found at the
 * weight cap (255) is taken to have reached it with this frame.
 * n_updated: if not NULL, synchronises and stores the voxels the frame
 * updated. */
VSG_API int vsg_integrate_backward(vsg_scene* s, const float* pointmap, int w, int h, float truncation,
                                   const float pose[16], float fx, float fy, float cx, float cy, float* grad_sdf,
                                   double* grad_pose, float* grad_pointmap, uint32_t* n_updated,
                                   vsg_stream_t stream);
/* Pool indices of the given blocks (host int32 coords[n*3] -> host int32
 * ptrs[n], -1 = not allocated): the row of grad_sdf, or of the voxel pool,
 * that holds each block.  Synchronises. */
VSG_API int vsg_scene_lookup_blocks(const vsg_scene* s, const int32_t* coords, uint32_t n, int32_t* ptrs);
/* Gauss-Newton normal equations of a weighted depth least-squares pose
 * problem on the last recorded render (no reference counterpart): with
 * J_i = d depth_i / d xi for the pose perturbation T exp(xi), xi = (omega,
 * v) (dR = R [omega]x, dt = R v), accumulates H = sum w_i J_i J_i^T and
 * b = sum w_i J_i r_i over hit pixels in double.  residual: device
 * float[w*h] (e.g. rendered minus observed depth); weights: device float[w*h]
 * (robust weights; NULL = 1; 0 leaves a pixel out).  normal_eq: DEVICE
 * double[27] receiving H's upper triangle row by row (21) then b (6); the
 * step is xi = -H^-1 b.  min_weight_sum and n_skipped as for
 * vsg_render_backward. */
VSG_API int vsg_render_pose_normal_equations(const vsg_renderer* r, const vsg_scene* s, const float pose[16],
                                             float fx, float fy, float cx, float cy, const float* residual,
                                             const float* weights, float min_weight_sum, double* normal_eq,
                                             uint32_t* n_skipped, vsg_stream_t stream);
/* Normals of the last recorded render (the reference never writes its normal
 * output): the normalised trilinear SDF gradient at each hit point, pointing
 * towards increasing SDF like computeNormalFromSDF (RayCastRender.cu:629-677);
 * misses get 1e10.  normals: device float4[w*h]. */
VSG_API int vsg_render_normals(const vsg_renderer* r, const vsg_scene* s, const float pose[16], float fx, float fy,
                               float cx, float cy, float* normals, uint32_t* n_skipped, vsg_stream_t stream);

/* ---- marching cubes -----------------------------------------------------
 * Replaces allocateMarchingCubesOutput / freeMarchingCubesOutput /
 * runMarchingCubesCUDA / copyMarchingCubesTriangleCount (MarchingCubes.h:
 * 34-58, MarchingCubes.cu:472-571).  Triangle soup over every allocated
 * block, cubes inside one block only, vertices float3[3 * max_triangles] and
 * per-vertex face normals float3[3 * max_triangles] on the device. */
typedef struct vsg_mc_output vsg_mc_output;

/* allocateMarchingCubesOutput: buffers for max_triangles triangles, on the
 * current device. */
VSG_API int vsg_mc_output_create(int max_triangles, vsg_mc_output** out);
/* freeMarchingCubesOutput */
VSG_API int vsg_mc_output_destroy(vsg_mc_output* m);
/* runMarchingCubesCUDA: extract the iso surface (iso: SDF level, 0 for the
 * surface; voxel_size <= 0 takes the scene's, as MarchingCubesParams'
 * voxelSize does).  Triangles go out in an unspecified order, each block's
 * as one range; the first max_triangles of them are written.
 * Stream-ordered; does not synchronise (the reference does). */
VSG_API int vsg_mc_run(vsg_scene* s, vsg_mc_output* m, float iso, float voxel_size, vsg_stream_t stream);
/* copyMarchingCubesTriangleCount: the surface's triangle count, which may
 * exceed the capacity (then only max_triangles were written).  Synchronises. */
VSG_API int vsg_mc_triangle_count(const vsg_mc_output* m, int64_t* count);
/* Device buffers (MarchingCubesOutput's d_vertices / d_normals /
 * d_triangleCount, the count as int clamped to INT_MAX); any pointer may be
 * NULL. */
VSG_API int vsg_mc_output_buffers(const vsg_mc_output* m, float** vertices, float** normals, int** count_dev,
                                  int* max_triangles);
/* Copy the written triangles to host memory: vertices / normals float[9 *
 * min(count, max_triangles)] (either may be NULL); count as in
 * vsg_mc_triangle_count.  Synchronises. */
VSG_API int vsg_mc_download(const vsg_mc_output* m, float* vertices, float* normals, int64_t* count);

/* ---- voxel-wise surface-point extraction ---------------------------------
 * Replaces RayCastRender::extractSurfacePoints / extractSurfacePointsCUDA /
 * saveExtractedSurfacePointsPLY (RayCastRender.h:91-109, RayCastRender.cu:
 * 683-910, RayCastRender.cpp:307-446).  One point per voxel with weight
 * >= max(1, min_weight) and SDF in [min_sdf, max_sdf] that has a zero
 * crossing towards a neighbour (or |sdf| < 0.001): float4 position (w = 1),
 * colour / 255 (w = 1) and SDF-gradient normal (w = 0), unspecified order. */
typedef struct vsg_points vsg_points;

/* buffers for max_points points on the current device (the reference
 * allocates 10,000,000) */
VSG_API int vsg_points_create(int max_points, vsg_points** out);
VSG_API int vsg_points_destroy(vsg_points* m);
/* Stream-ordered; does not synchronise. */
VSG_API int vsg_extract_points(vsg_scene* s, vsg_points* m, float min_sdf, float max_sdf, uint32_t min_weight,
                               vsg_stream_t stream);
/* The number of points found, which may exceed the capacity (then only
 * max_points were written).  Synchronises. */
VSG_API int vsg_points_count(const vsg_points* m, int64_t* count);
/* Device buffers (float4 each; the count as int clamped to INT_MAX). */
VSG_API int vsg_points_buffers(const vsg_points* m, float** positions, float** colors, float** normals,
                               int** count_dev, int* max_points);
/* Copy the written points to host float4 arrays (any may be NULL). */
VSG_API int vsg_points_download(const vsg_points* m, float* positions, float* colors, float* normals,
                                int64_t* count);
/* ASCII PLY as saveExtractedSurfacePointsPLY writes it. */
VSG_API int vsg_points_save_ply(const vsg_points* m, const char* path);

/* ---- streaming between the scene and host memory -------------------------
 * Replaces VoxelStreamingManager (VoxelStreamingManager.h:140-301): the
 * host-side chunk grid (m_grid, :246) is a vsg_block_store; stream out =
 * streamOutFindBlocksOnGPU + streamOutCopyToChunkGrid (VoxelStreamingManager.
 * cpp:303-527), stream in = streamInCopyToGPUBuffer + streamInInsertToHashTable
 * (:530-834).  Both synchronise.  Differences: stream-in really inserts (the
 * reference's insertion is switched off), a block that is resident or stored
 * twice is merged voxel by voxel (weights add, capped at 255; SDF and colour
 * weight-averaged), no per-call cap and no chunk-grid bounds. */
typedef struct vsg_block_store vsg_block_store;

/* chunk_extent: g_streamingVoxelExtents (m, NULL = 1 m cubes). */
VSG_API int vsg_store_create(const float chunk_extent[3], vsg_block_store** out);
VSG_API int vsg_store_destroy(vsg_block_store* st);
VSG_API int vsg_store_info(const vsg_block_store* st, uint64_t* n_blocks, uint64_t* n_chunks);
/* Stored blocks as vsg_scene_export lays them out (sorted coords, 8-byte
 * voxels; voxels may be NULL).  VSG_ERR_TOO_LARGE when more than max_blocks. */
VSG_API int vsg_store_export(const vsg_block_store* st, int32_t* coords, uint8_t* voxels, uint64_t max_blocks,
                             uint64_t* n_out);
/* Checkpoint file of the stored blocks in the reference's streaming record
 * layout (SDFBlockInfo + SDFBlock of 12-byte VoxelData, VoxelStreamingManager.h:
 * 30-76) after a 32-byte header; load merges the file into the store. */
VSG_API int vsg_store_save(const vsg_block_store* st, const char* path);
VSG_API int vsg_store_load(vsg_block_store* st, const char* path);
/* How many stored blocks (in how many chunks) a vsg_stream_in with this
 * centre and radius would take (VoxelStreamingManager::streamInFindChunk,
 * VoxelStreamingManager.cpp:993-1140, which returns the block count);
 * radius < 0: everything stored. */
VSG_API int vsg_store_count(const vsg_block_store* st, const float center[3], float radius, uint64_t* n_blocks,
                            uint64_t* n_chunks);
/* File n host blocks given in the reference's streaming records
 * (VoxelStreamingManager::updateChunkGrid, VoxelStreamingManager.cpp:836-903):
 * infos = n SDFBlockInfo {int3 pos, int ptr} (4 int32 each), voxels = n
 * SDFBlock of 512 12-byte VoxelData {uchar3 colour, uchar weight, float sdf,
 * 2 flag bytes, 2 pad}; blocks already stored merge as in stream-out.
 * voxel_size must match the blocks already held. */
VSG_API int vsg_store_add_records(vsg_block_store* st, float voxel_size, const int32_t* infos,
                                  const uint8_t* voxels, uint64_t n);
/* Move every block whose corner lies at distance >= radius from center into
 * the store (deleted from the scene, pool blocks freed). */
VSG_API int vsg_stream_out(vsg_scene* s, vsg_block_store* st, const float center[3], float radius, uint32_t* n_out,
                           vsg_stream_t stream);
/* Move the stored chunks that intersect the sphere back into the scene
 * (radius < 0: every stored block).  VSG_ERR_TOO_LARGE, with nothing moved,
 * when the free pool cannot hold them. */
VSG_API int vsg_stream_in(vsg_scene* s, vsg_block_store* st, const float center[3], float radius, uint32_t* n_in,
                          uint32_t* n_merged, vsg_stream_t stream);
/* Whole-scene checkpoint in the same file format (no counterpart in the
 * reference): save writes every allocated block; load inserts the file's
 * blocks (merging into resident ones). */
VSG_API int vsg_scene_save(vsg_scene* s, const char* path);
VSG_API int vsg_scene_load(vsg_scene* s, const char* path, vsg_stream_t stream);

/* ---- batched form: many independent scenes advanced together ----------
 * No counterpart in the reference (it fuses one scan at a time).  A batch
 * holds up to 256 scenes (each its own hash table and voxel pool, any
 * resolution) and optional per-scene renderers.  vsg_batch_step integrates
 * one frame for each listed scene -- and ray casts it at the same pose when
 * `render` is set -- with one launch per stage for all of them; the step's
 * launch sequence is captured into a CUDA graph and replayed while the set
 * of resolutions stays the same.  Every scene's results are identical to
 * vsg_integrate followed by vsg_render. */
typedef struct vsg_batch vsg_batch;

typedef struct vsg_batch_frame {
    int scene;              /* index into the scenes given to vsg_batch_create */
    const float* pointmap;  /* device float3[w*h] camera-space points */
    const uint8_t* rgb;     /* device uchar3[w*h] */
    const float* normals;   /* device float3[w*h] (not read; must be non-null) */
    int w, h;
    float truncation;
    float pose[16];         /* row-major camera->world (copied at the call) */
    float fx, fy, cx, cy;
    float min_depth, max_depth; /* ray cast range */
    int render;             /* 1: ray cast into the scene's renderer (w x h) */
} vsg_batch_frame;

VSG_API int vsg_batch_create(vsg_scene* const* scenes, vsg_renderer* const* renderers, int n, vsg_batch** out);
VSG_API int vsg_batch_destroy(vsg_batch* b);
/* Each scene at most once per step.  The first step of a new shape runs
 * eagerly (and, with autotuning on, times five ray-cast launch variants, 4
 * to 8 resident CTAs per SM, on its own data) and captures the graph; later steps replay it. */
VSG_API int vsg_batch_step(vsg_batch* b, const vsg_batch_frame* frames, int n_frames, vsg_stream_t stream);
VSG_API int vsg_batch_autotune(vsg_batch* b, int enable);

/* Per-kernel device time (ms) since the last vsg_timing_reset, measured
 * with CUDA events on the launching stream when timing is enabled.
 * Slots: 0 alloc, 1 integrate, 2 render, 3 select, 4 marching cubes,
 * 5 surface-point extraction.
 * counts[i] = launches. */
VSG_API int vsg_timing_enable(vsg_scene* s, int enable);
VSG_API int vsg_timing_read(vsg_scene* s, double* ms, uint32_t* counts, int n_slots);
VSG_API int vsg_timing_reset(vsg_scene* s);

/* March statistics of this scene's renders (off by default): with enable
 * != 0 vsg_render / vsg_render_hostpose also count the samples skipped as
 * empty, the samples taken at a skip-cell boundary and the distinct blocks
 * the rays read (vsg_stats.render_samples_skipped, render_singles,
 * render_blocks_read; 0 while off).  The outputs are the same either way;
 * the counting ray caster is about 10 % slower.  Batched steps never count
 * them. */
VSG_API int vsg_scene_march_stats(vsg_scene* s, int enable);

/* Library version string. */
VSG_API const char* vsg_version(void);

#ifdef __cplusplus
}
#endif

#endif /* VSG_H */
