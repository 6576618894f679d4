/*
 * voxelsg_b200.hpp -- header-only C++ drop-in for VoxelSG's fusion API over
 * the C ABI of libvsg.so (vsg.h).
 *
 * Keeps the reference names, signatures and error behaviour of
 *   GlobalParamsConfig   (globalPramasConfig.h:55-187; defaults
 *                         globalParamasConfig.cpp:8-402; validation :413-417)
 *   Params               (CUDAHashData.h:9-42, including its swap of the two
 *                         truncation fields, CUDAHashData.h:27-28)
 *   VoxelScene           (VoxelScene.h:51-209): constructor, reset,
 *                         integrateFromScanData, getNumIntegratedFrames,
 *                         isAllocated, getParams, getHeapFreeCount,
 *                         compactifyHashEntries, printStats, saveToMesh,
 *                         getOutputDirectory
 *   RayCastRender        (RayCastRender.h:20-124): initialize, render,
 *                         downloadResults, downloadDepthFloat, savePointCloudPLY,
 *                         getOutputDepth/Color/Normal/Positions,
 *                         extractSurfacePoints, saveExtractedSurfacePointsPLY
 *   MarchingCubesParams, MarchingCubesOutput, allocateMarchingCubesOutput,
 *   freeMarchingCubesOutput, runMarchingCubesCUDA,
 *   copyMarchingCubesTriangleCount (MarchingCubes.h:7-58)
 *   VoxelStreamingManager (VoxelStreamingManager.h:140-301): constructor,
 *                         streamOut / streamIn, streamOutFindBlocksOnGPU,
 *                         streamOutCopyToChunkGrid, streamInCopyToGPUBuffer,
 *                         streamInInsertToHashTable
 *   CustomDepthMapGenerator (CustomDepthMapGenerator.h:15-165): setCameraParams,
 *                         setProjectionMethod, generateFromPointCloud
 * so that reference call sites compile unchanged against it.  Like the
 * reference, the methods print to stderr and return on bad input instead of
 * throwing; the only throw is GlobalParamsConfig::initialize.
 *
 * cv::Mat is not required: integrateFromScanData accepts any 4x4 matrix type
 * with at<float>(row, col) (cv::Mat, or vsg::Mat4f below).
 */
#pragma once

#include <cuda_runtime.h>
#include <vector_types.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "vsg.h"

#ifndef SDF_BLOCK_SIZE
#define SDF_BLOCK_SIZE 8
#endif
#ifndef HASH_BUCKET_SIZE
#define HASH_BUCKET_SIZE 10
#endif

namespace vsg {

/* Row-major 4x4 float matrix with the cv::Mat accessor the API uses. */
struct Mat4f {
    float m[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    template <class T>
    T& at(int r, int c) {
        return m[r * 4 + c];
    }
    template <class T>
    const T& at(int r, int c) const {
        return m[r * 4 + c];
    }
};

}  // namespace vsg

/* The reference's small vector types (its utils.h); define VSG_HAVE_VEC3
 * before including this header to use your own. */
#ifndef VSG_HAVE_VEC3
struct vec3f {
    float x = 0.0f, y = 0.0f, z = 0.0f;
    vec3f() = default;
    vec3f(float a, float b, float c) : x(a), y(b), z(c) {}
};
struct vec3i {
    int x = 0, y = 0, z = 0;
    vec3i() = default;
    vec3i(int a, int b, int c) : x(a), y(b), z(c) {}
};
struct vec4f {
    float x = 0.0f, y = 0.0f, z = 0.0f, w = 0.0f;
    vec4f() = default;
    vec4f(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
};
#endif

/* The knobs the fusion path reads, with the reference's code defaults. */
class GlobalParamsConfig {
public:
    /* Every knob of globalPramasConfig.h:55-170 with the defaults of
     * globalParamasConfig.cpp:8-402.  The fusion path reads the SDF, hash,
     * marching-cubes and streaming knobs; the sensor, texture, rendering,
     * tracking and recording knobs belong to parts of the reference outside
     * this library and are kept only so that code setting them compiles. */
    std::string g_data_name;
    unsigned int g_sensorIdx = 0;
    std::string g_sceneName;
    std::string g_binaryDumpSensorFile0;
    unsigned int g_optimizationIdx = 0;
    int g_gain = 1;
    int g_exposure = 200;
    bool g_autoExposureEnabled = false;
    bool g_autoWhiteBalanceEnabled = false;
    bool g_renderToFile = false;
    bool g_voxelRenderingEnabled = false;
    unsigned int g_texKeyFrames = 4;
    int g_nVideoFrame = 900;
    int g_startFrame = 0;
    unsigned int g_texPoolPatchWidth = 4;
    unsigned int g_texPoolNumPatches = 1000000;
    unsigned int g_numTextureTileWidth = 1024;
    unsigned int g_texIntegrationWeightMax = 255;
    unsigned int g_texIntegrationWeightSample = 30;
    float g_erodeSigmaStretch = 2.0f;
    unsigned int g_erodeIterStretchBox = 0;
    unsigned int g_erodeIterStretchGauss = 0;
    unsigned int g_erodeIterOccDepth = 6;
    float g_texAngleThreshold_depth = 0.05f;
    float g_texAngleThreshold_update = 0.5f;
    float g_screenBoundaryWidth = 40.0f;
    float g_sigmaAngle = 0.5f;
    float g_sigmaDepth = 0.5f;
    float g_sigmaArea = 1.0f;
    unsigned int g_windowWidth = 640;
    unsigned int g_windowHeight = 480;
    unsigned int g_adapterWidth = 640;
    unsigned int g_adapterHeight = 480;
    float g_sensorDepthMax = 3.0f;
    float g_sensorDepthMin = 0.4f;
    bool g_enableColorCropping = false;
    unsigned int g_colorCropX = 320;
    unsigned int g_colorCropY = 272;
    unsigned int g_colorCropWidth = 640;
    unsigned int g_colorCropHeight = 480;
    float g_SDFVoxelSize = 0.1f;          /* globalParamasConfig.cpp:28 */
    float g_SDFMarchingCubeThreshFactor = 10.0f;
    float g_SDFTruncation = 0.25f;        /* :38 */
    float g_SDFTruncationScale = 0.01f;   /* :44 */
    float g_SDFMaxIntegrationDistance = 3.0f;
    unsigned int g_SDFIntegrationWeightSample = 3;
    unsigned int g_SDFIntegrationWeightMax = 255;
    unsigned int g_hashNumSlots = 10000;  /* :61 */
    unsigned int g_hashNumSDFBlocks = 10000; /* :65 */
    unsigned int g_hashMaxCollisionLinkedListSize = 5;
    unsigned int g_hashSlotSize = HASH_BUCKET_SIZE;
    unsigned int g_hashNumBuckets = 10000; /* = g_hashNumSlots, :74 */
    float g_SDFRayIncrementFactor = 0.8f;
    float g_SDFRayThresSampleDistFactor = 50.5f;
    float g_SDFRayThresDistFactor = 50.0f;
    bool g_SDFUseGradients = false;
    bool g_binaryDumpSensorUseTrajectory = false;
    bool g_binaryDumpSensorUseTrajectoryOnlyInit = false;
    float g_depthSigmaD = 2.0f;
    float g_depthSigmaR = 0.1f;
    bool g_depthFilter = true;
    float g_colorSigmaD = 1.0f;
    float g_colorSigmaR = 0.08f;
    bool g_colorFilter = false;
    vec4f g_materialAmbient = vec4f(0.75f, 0.65f, 0.5f, 1.0f);
    vec4f g_materialSpecular = vec4f(1.0f, 1.0f, 1.0f, 1.0f);
    vec4f g_materialDiffuse = vec4f(1.0f, 0.9f, 0.7f, 1.0f);
    float g_materialShininess = 16.0f;
    vec4f g_lightAmbient = vec4f(0.4f, 0.4f, 0.4f, 1.0f);
    vec4f g_lightDiffuse = vec4f(0.6f, 0.52944f, 0.4566f, 0.6f);
    vec4f g_lightSpecular = vec4f(0.3f, 0.3f, 0.3f, 1.0f);
    vec3f g_lightDirection = vec3f(0.0f, -1.0f, 2.0f);
    unsigned int g_RnderMode = 1;
    bool g_useColorForRendering = false;
    bool g_playData = true;
    float g_renderingDepthDiscontinuityThresLin = 0.001f;
    float g_rmappingDepthDiscontinuityThresLin = 0.0f;
    float g_renderingDepthDiscontinuityThresOffset = 0.012f;
    float g_remappingDepthDiscontinuityThresOffset = 0.0f;
    bool g_bUseCameraCalibration = false;
    unsigned int g_marchingCubesMaxNumTriangles = 250000; /* :379 */
    bool g_streamingEnabled = true;       /* :119 */
    vec3f g_streamingVoxelExtents = vec3f(1.0f, 1.0f, 1.0f);        /* :124 */
    vec3i g_streamingGridDimensions = vec3i(513, 513, 513);         /* :127 */
    vec3i g_streamingMinGridPos = vec3i(-256, -256, -256);          /* :130 */
    unsigned int g_streamingInitialChunkListSize = 2000;            /* :133 */
    float g_streamingRadius = 4.0f;       /* :136 */
    vec3f g_streamingPos = vec3f(0.0f, 0.0f, 3.0f);
    unsigned int g_streamingOutParts = 80;
    bool g_recordData = false;
    bool g_recordCompression = true;
    std::string g_recordDataFile = "Dump/test.sens";
    bool g_reconstructionEnabled = true;
    bool g_offlineProcessing = false;
    bool g_integrationEnabled = true;
    bool g_trackingEnabled = true;
    bool g_timingsDetailledEnabled = false;
    bool g_timingsDetailledEnabledOurs = false;
    bool g_timingsTotalEnabled = false;
    bool g_garbageCollectionEnabled = false;
    unsigned int g_garbageCollectionStarve = 15;
    int g_warpingMode = 0;
    int g_depth_map_H = 400;
    int g_depth_map_W = 480;
    int g_maxDirectionalSlots = 0;
    float g_directionThresholdCosine = 0.0f;
    float g_weightMax = 0.0f;

    /* globalParamasConfig.cpp:8-402 */
    void setDefault() { *this = GlobalParamsConfig(); }
    void print() const {
        std::cout << "GlobalParamsConfig: voxel " << g_SDFVoxelSize << " m, truncation " << g_SDFTruncation
                  << " m (scale " << g_SDFTruncationScale << "), hash slots " << g_hashNumSlots << ", SDF blocks "
                  << g_hashNumSDFBlocks << ", marching cubes max triangles " << g_marchingCubesMaxNumTriangles
                  << ", streaming " << (g_streamingEnabled ? "on" : "off") << std::endl;
    }

    static GlobalParamsConfig& getInstance() {
        static GlobalParamsConfig s;
        return s;
    }
    static GlobalParamsConfig& get() { return getInstance(); }

    void initialize() {
        validateParameters();
        m_bIsInitialized = true;
    }
    bool isInitialized() const { return m_bIsInitialized; }
    void validateParameters() const {
        if (g_hashNumBuckets == 0) throw std::invalid_argument("Invalid hash buckets");
        if (g_SDFVoxelSize <= 0.0f) throw std::invalid_argument("Invalid voxel size");
    }

private:
    bool m_bIsInitialized = false;
};

/* Params derived from the knobs (CUDAHashData.h:14-29). */
struct Params {
    Params() = default;
    explicit Params(const GlobalParamsConfig& gpc) {
        SDFBlockNum = (int)gpc.g_hashNumSDFBlocks;
        hashSlotNum = (int)gpc.g_hashNumSlots;
        SDFBlockSize = SDF_BLOCK_SIZE;
        slotSize = HASH_BUCKET_SIZE;
        totalHashSize = (int)gpc.g_hashNumSlots * HASH_BUCKET_SIZE;
        totalBlockSize = (int)gpc.g_hashNumSDFBlocks * SDF_BLOCK_SIZE * SDF_BLOCK_SIZE * SDF_BLOCK_SIZE;
        voxelSize = gpc.g_SDFVoxelSize;
        truncationScale = gpc.g_SDFTruncation;   /* the reference swaps these two */
        truncation = gpc.g_SDFTruncationScale;
    }
    int hashSlotNum = 0;
    int SDFBlockNum = 0;
    int SDFBlockSize = SDF_BLOCK_SIZE;
    int totalHashSize = 0;
    int slotSize = HASH_BUCKET_SIZE;
    int totalBlockSize = 0;
    float voxelSize = 0.0f;
    float truncationScale = 0.0f;
    float truncation = 0.0f;
};

class VoxelScene;

/* What VoxelScene::getHashData hands to the marching-cubes launcher: here a
 * view of the scene's handle (the reference exposes its raw hash arrays). */
struct CUDAHashRef {
    vsg_scene* scene = nullptr;
};

class VoxelScene {
public:
    explicit VoxelScene(const Params& params) : m_params(params) {
        vsg_params p;
        vsg_params_default(&p);
        p.voxel_size = params.voxelSize;
        p.truncation = params.truncationScale;
        p.truncation_scale = params.truncation;
        p.hash_num_slots = (uint32_t)params.hashSlotNum;
        p.num_sdf_blocks = (uint32_t)params.SDFBlockNum;
        const int rc = vsg_scene_create(&p, &m_scene);
        if (rc != VSG_OK) {
            std::cerr << "VoxelScene: allocation failed (status " << rc << ")" << std::endl;
            m_scene = nullptr;
        }
#ifdef USE_NORMAL_DIR_ALLOC
        // the reference's compile-time switch (VoxelScene.cu:8, 1688)
        if (m_scene) vsg_scene_set_alloc_method(m_scene, 2);
#endif
    }
    ~VoxelScene() {
        if (m_scene) vsg_scene_destroy(m_scene);
    }
    VoxelScene(const VoxelScene&) = delete;
    VoxelScene& operator=(const VoxelScene&) = delete;

    void reset() {
        if (!m_scene) {
            std::cerr << "VoxelScene: Not allocated yet!" << std::endl;
            return;
        }
        vsg_scene_reset(m_scene, nullptr);
        cudaDeviceSynchronize();
    }

    /* VoxelScene.h:89-91.  depthmap / colormap / normalmap are device maps;
     * cameraTransform is a host 4x4 camera->world matrix. */
    template <class Matrix>
    void integrateFromScanData(const float3* depthmap, const uchar3* colormap, const float3* normalmap, int width,
                               int height, float truncationDistance, const Matrix& cameraTransform, float fx,
                               float fy, float cx, float cy) {
        if (depthmap == nullptr || colormap == nullptr || normalmap == nullptr) {
            std::cerr << "VoxelScene: Invalid pointers (nullptr)!" << std::endl;
            return;
        }
        if (!m_scene) {
            std::cerr << "VoxelScene: Not allocated!" << std::endl;
            return;
        }
        float T[16];
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) T[i * 4 + j] = cameraTransform.template at<float>(i, j);
        const int rc = vsg_integrate(m_scene, reinterpret_cast<const float*>(depthmap),
                                     reinterpret_cast<const uint8_t*>(colormap),
                                     reinterpret_cast<const float*>(normalmap), width, height, truncationDistance,
                                     T, fx, fy, cx, cy, nullptr);
        if (rc != VSG_OK) std::cerr << "VoxelScene: integration failed (status " << rc << ")" << std::endl;
    }

    unsigned int getNumIntegratedFrames() const {
        vsg_stats st{};
        if (!m_scene || vsg_scene_stats(m_scene, &st) != VSG_OK) return 0;
        return st.integrated_frames;
    }
    /* VoxelScene.cpp:348-354: heap counter + 1 = free blocks */
    unsigned int getHeapFreeCount() const {
        vsg_stats st{};
        if (!m_scene || vsg_scene_stats(m_scene, &st) != VSG_OK) return 0;
        return st.free_blocks;
    }
    bool isAllocated() const { return m_scene != nullptr; }
    /* VoxelScene.h:97: the reference lists every allocated block here;
     * vsg_integrate selects the blocks a frame can touch itself, so there is
     * nothing to do between frames. */
    void compactifyHashEntries() {}
    /* VoxelScene.cpp:380-398 */
    void printStats() const {
        std::cout << "\n=== VoxelScene Stats ===" << std::endl;
        std::cout << "Hash Slots: " << m_params.hashSlotNum << std::endl;
        std::cout << "Bucket Size: " << m_params.slotSize << std::endl;
        std::cout << "Total Hash Entries: " << m_params.totalHashSize << std::endl;
        std::cout << "SDF Blocks: " << m_params.SDFBlockNum << std::endl;
        std::cout << "Block Size: " << m_params.SDFBlockSize << "x" << m_params.SDFBlockSize << "x"
                  << m_params.SDFBlockSize << std::endl;
        std::cout << "Total Voxels: " << m_params.totalBlockSize << std::endl;
        std::cout << "Integrated Frames: " << getNumIntegratedFrames() << std::endl;
        if (m_scene) {
            const unsigned int freeCount = getHeapFreeCount();
            std::cout << "Free Blocks: " << freeCount << " / " << m_params.SDFBlockNum << " ("
                      << (freeCount * 100.0 / (m_params.SDFBlockNum ? m_params.SDFBlockNum : 1)) << "%)"
                      << std::endl;
        }
        std::cout << "========================\n" << std::endl;
    }
    /* VoxelScene.cpp:838-845 is a stub that returns false.  Here: marching
     * cubes over the scene (iso 0, up to maxTriangles) written as an ASCII PLY
     * mesh (vertices, then faces of three consecutive vertices); false when
     * the scene is empty, the file cannot be written or a call fails. */
    bool saveToMesh(const std::string& filename, int maxTriangles = 4000000) {
        if (!m_scene || maxTriangles <= 0) return false;
        vsg_mc_output* mc = nullptr;
        if (vsg_mc_output_create(maxTriangles, &mc) != VSG_OK) return false;
        bool ok = vsg_mc_run(m_scene, mc, 0.0f, m_params.voxelSize, nullptr) == VSG_OK;
        int64_t n = 0;
        std::vector<float> v, nrm;
        if (ok) ok = vsg_mc_download(mc, nullptr, nullptr, &n) == VSG_OK;
        const int64_t k = n < maxTriangles ? n : maxTriangles;
        if (ok && k > 0) {
            v.resize((size_t)k * 9);
            nrm.resize((size_t)k * 9);
            ok = vsg_mc_download(mc, v.data(), nrm.data(), &n) == VSG_OK;
        }
        vsg_mc_output_destroy(mc);
        if (!ok || k <= 0) return false;
        FILE* f = std::fopen(filename.c_str(), "w");
        if (!f) return false;
        std::fprintf(f, "ply\nformat ascii 1.0\nelement vertex %lld\nproperty float x\nproperty float y\n"
                        "property float z\nelement face %lld\nproperty list uchar int vertex_indices\nend_header\n",
                     (long long)(3 * k), (long long)k);
        for (int64_t i = 0; i < 3 * k; ++i) std::fprintf(f, "%g %g %g\n", v[3 * i], v[3 * i + 1], v[3 * i + 2]);
        for (int64_t t = 0; t < k; ++t)
            std::fprintf(f, "3 %lld %lld %lld\n", (long long)(3 * t), (long long)(3 * t + 1), (long long)(3 * t + 2));
        return std::fclose(f) == 0;
    }
    /* VoxelScene.h:148: the reference's per-run log directory; logs are not
     * written here, so this is the current directory. */
    std::string getOutputDirectory() const { return "."; }
    Params& getParams() { return m_params; }
    const Params& getParams() const { return m_params; }
    vsg_scene* handle() const { return m_scene; }
    /* VoxelScene.h:129 */
    CUDAHashRef& getHashData() {
        m_hashRef.scene = m_scene;
        return m_hashRef;
    }

private:
    Params m_params;
    vsg_scene* m_scene = nullptr;
    CUDAHashRef m_hashRef;
};

class RayCastRender {
public:
    RayCastRender() = default;
    ~RayCastRender() {
        if (m_r) vsg_renderer_destroy(m_r);
        if (m_points) vsg_points_destroy(m_points);
    }
    RayCastRender(const RayCastRender&) = delete;
    RayCastRender& operator=(const RayCastRender&) = delete;

    bool initialize(int width, int height) {
        if (m_r) {
            std::cerr << "RayCastRender: Already initialized!" << std::endl;
            return false;
        }
        if (vsg_renderer_create(width, height, &m_r) != VSG_OK) {
            std::cerr << "RayCastRender: Failed to allocate GPU memory!" << std::endl;
            m_r = nullptr;
            return false;
        }
        m_width = width;
        m_height = height;
        return true;
    }

    /* RayCastRender.h:66-70: cameraTransform is a DEVICE float[16]
     * (row-major camera->world); cameraPos is the ray origin. */
    void render(const VoxelScene* voxelScene, float3 cameraPos, float* cameraTransform, float fx, float fy, float cx,
                float cy, float minDepth, float maxDepth) {
        if (!m_r) {
            std::cerr << "RayCastRender: Not initialized!" << std::endl;
            return;
        }
        if (!voxelScene || !voxelScene->isAllocated()) {
            std::cerr << "RayCastRender: Invalid voxel scene!" << std::endl;
            return;
        }
        const float cam[3] = {cameraPos.x, cameraPos.y, cameraPos.z};
        const int rc = vsg_render(m_r, voxelScene->handle(), cam, cameraTransform, fx, fy, cx, cy, minDepth,
                                  maxDepth, nullptr);
        if (rc != VSG_OK) std::cerr << "RayCastRender: render failed (status " << rc << ")" << std::endl;
        cudaDeviceSynchronize();
    }

    /* RayCastRender.cpp:188-212: depth expanded to (d, d, d, 1) */
    void downloadResults(float4* h_outputDepth, float4* h_outputColor, float4* h_outputNormal) {
        if (!m_r) {
            std::cerr << "RayCastRender: Not initialized!" << std::endl;
            return;
        }
        const size_t n = (size_t)m_width * m_height;
        std::vector<float> d(n);
        if (vsg_renderer_download(m_r, d.data(), nullptr, reinterpret_cast<float*>(h_outputColor),
                                  reinterpret_cast<float*>(h_outputNormal)) != VSG_OK) {
            std::cerr << "RayCastRender: Failed to download results!" << std::endl;
            return;
        }
        for (size_t i = 0; i < n; ++i) h_outputDepth[i] = make_float4(d[i], d[i], d[i], 1.0f);
    }

    void downloadDepthFloat(float* h_outputDepthFloat) {
        if (!m_r || h_outputDepthFloat == nullptr) return;
        vsg_renderer_download(m_r, h_outputDepthFloat, nullptr, nullptr, nullptr);
    }

    bool savePointCloudPLY(const std::string& filePath) {
        if (!m_r) {
            std::cerr << "RayCastRender: Not initialized!" << std::endl;
            return false;
        }
        int64_t n = 0;
        if (vsg_renderer_save_ply(m_r, filePath.c_str(), &n) != VSG_OK) {
            std::cerr << "RayCastRender: No valid raycast points to export." << std::endl;
            return false;
        }
        std::cout << "RayCastRender: Saved point cloud to " << filePath << " (" << n << " points)" << std::endl;
        return true;
    }

    /* the depth buffer holds floats although typed float4*, as in the
     * reference (RayCastRender.cpp:98, 151) */
    float4* getOutputDepth() const { return ptr(0); }
    float4* getOutputColor() const { return ptr(2); }
    float4* getOutputNormal() const { return ptr(3); }
    float4* getOutputPositions() const { return ptr(1); }
    int getWidth() const { return m_width; }
    int getHeight() const { return m_height; }
    bool isAllocated() const { return m_r != nullptr; }

    /* RayCastRender.cpp:307-360: point buffers (10,000,000 points, as the
     * reference) are created on the first call; returns the number found. */
    int extractSurfacePoints(const VoxelScene* voxelScene, float minSDF = -0.01f, float maxSDF = 0.01f,
                             unsigned int minWeight = 1) {
        if (!voxelScene || !voxelScene->isAllocated()) {
            std::cerr << "RayCastRender::extractSurfacePoints: Invalid voxelScene!" << std::endl;
            return 0;
        }
        if (!m_points && vsg_points_create(m_maxExtractedPoints, &m_points) != VSG_OK) {
            std::cerr << "RayCastRender::extractSurfacePoints: Failed to allocate GPU memory!" << std::endl;
            m_points = nullptr;
            return 0;
        }
        int64_t n = 0;
        if (vsg_extract_points(voxelScene->handle(), m_points, minSDF, maxSDF, minWeight, nullptr) != VSG_OK ||
            vsg_points_count(m_points, &n) != VSG_OK)
            return 0;
        m_numExtractedPoints = n > m_maxExtractedPoints ? m_maxExtractedPoints : (int)n;
        return m_numExtractedPoints;
    }
    bool saveExtractedSurfacePointsPLY(const std::string& filePath) {
        if (!m_points || m_numExtractedPoints == 0) {
            std::cerr << "RayCastRender::saveExtractedSurfacePointsPLY: No points to save!" << std::endl;
            return false;
        }
        return vsg_points_save_ply(m_points, filePath.c_str()) == VSG_OK;
    }
    float4* getExtractedPositions() const { return pts(0); }
    float4* getExtractedColors() const { return pts(1); }
    float4* getExtractedNormals() const { return pts(2); }
    int getNumExtractedPoints() const { return m_numExtractedPoints; }

private:
    float4* ptr(int which) const {
        if (!m_r) return nullptr;
        float* p[4] = {nullptr, nullptr, nullptr, nullptr};
        vsg_renderer_outputs(m_r, &p[0], &p[1], &p[2], &p[3]);
        return reinterpret_cast<float4*>(p[which]);
    }
    float4* pts(int which) const {
        if (!m_points) return nullptr;
        float* p[3] = {nullptr, nullptr, nullptr};
        vsg_points_buffers(m_points, &p[0], &p[1], &p[2], nullptr, nullptr);
        return reinterpret_cast<float4*>(p[which]);
    }
    vsg_renderer* m_r = nullptr;
    int m_width = 0, m_height = 0;
    vsg_points* m_points = nullptr;
    int m_maxExtractedPoints = 10000000;
    int m_numExtractedPoints = 0;
};

/* MarchingCubes.h:7-17 */
struct MarchingCubesParams {
    float isoValue = 0.0f;
    float voxelSize = 1.0f; /* > 0 overrides the scene's voxel size, as in the reference */
    int maxTriangles = 0;
};

/* MarchingCubes.h:19-31: device triangle soup (3 vertices / normals each). */
struct MarchingCubesOutput {
    float3* d_vertices = nullptr;
    float3* d_normals = nullptr;
    int* d_triangleCount = nullptr;
    int maxTriangles = 0;
    vsg_mc_output* handle = nullptr;
};

inline void freeMarchingCubesOutput(MarchingCubesOutput& output) {
    if (output.handle) vsg_mc_output_destroy(output.handle);
    output = MarchingCubesOutput();
}

inline void allocateMarchingCubesOutput(MarchingCubesOutput& output, int maxTriangles) {
    if (maxTriangles <= 0) {
        std::cerr << "allocateMarchingCubesOutput: maxTriangles must be positive." << std::endl;
        return;
    }
    freeMarchingCubesOutput(output);
    if (vsg_mc_output_create(maxTriangles, &output.handle) != VSG_OK) {
        std::cerr << "allocateMarchingCubesOutput: allocation failed" << std::endl;
        output.handle = nullptr;
        return;
    }
    float *v = nullptr, *n = nullptr;
    vsg_mc_output_buffers(output.handle, &v, &n, &output.d_triangleCount, &output.maxTriangles);
    output.d_vertices = reinterpret_cast<float3*>(v);
    output.d_normals = reinterpret_cast<float3*>(n);
}

/* The reference synchronises the stream before returning; so does this. */
inline void runMarchingCubesCUDA(const CUDAHashRef& hashData, const Params& params,
                                 const MarchingCubesParams& paramsMC, MarchingCubesOutput& output,
                                 cudaStream_t stream = nullptr) {
    (void)params; /* the scene carries its own voxel size */
    if (hashData.scene == nullptr) {
        std::cerr << "runMarchingCubesCUDA: Hash data not initialized." << std::endl;
        return;
    }
    if (output.handle == nullptr) {
        std::cerr << "runMarchingCubesCUDA: Output buffers not allocated." << std::endl;
        return;
    }
    if (vsg_mc_run(hashData.scene, output.handle, paramsMC.isoValue, paramsMC.voxelSize, stream) != VSG_OK) {
        std::cerr << "runMarchingCubesCUDA: kernel launch failed" << std::endl;
        return;
    }
    if (cudaStreamSynchronize(stream) != cudaSuccess)
        std::cerr << "runMarchingCubesCUDA: stream sync failed" << std::endl;
}

inline int copyMarchingCubesTriangleCount(const MarchingCubesOutput& output) {
    int64_t n = 0;
    if (!output.handle || vsg_mc_triangle_count(output.handle, &n) != VSG_OK) return 0;
    return n > 2147483647 ? 2147483647 : (int)n;
}

/* VoxelStreamingManager.h:140-301 over vsg_stream_* and a vsg_block_store.
 * Single host thread: the reference's auxiliary thread and its Win32 event
 * handshakes are not reproduced (the multiThreaded flags are accepted and
 * ignored), streamOutFindBlocksOnGPU already files the blocks in the host
 * chunk grid (streamOutCopyToChunkGrid has nothing left to do), and
 * streamInCopyToGPUBuffer only records the sphere that
 * streamInInsertToHashTable then brings back.  The chunk grid has no bounds
 * (gridDimensions / minGridPos are accepted, not enforced). */
class VoxelStreamingManager {
public:
    VoxelStreamingManager(VoxelScene& sceneHashRef, Params& params, const vec3f& voxelExtends,
                          const vec3i& gridDimensions, const vec3i& minGridPos, unsigned int initialChunkListSize,
                          bool streamingEnabled)
        : m_scene(&sceneHashRef), m_params(params) {
        initialize(voxelExtends, gridDimensions, minGridPos, initialChunkListSize, streamingEnabled);
    }
    /* VoxelStreamingManager.cpp:136-166: a fresh, empty chunk grid.  The
     * store has no grid bounds; the dimensions only serve the chunk helpers
     * below. */
    void initialize(const vec3f& voxelExtends, const vec3i& gridDimensions, const vec3i& minGridPos,
                    unsigned int initialChunkListSize, bool streamingEnabled) {
        (void)initialChunkListSize;
        (void)streamingEnabled;
        if (m_store) vsg_store_destroy(m_store);
        m_store = nullptr;
        m_ext = voxelExtends;
        m_dims = gridDimensions;
        m_min = minGridPos;
        const float e[3] = {voxelExtends.x, voxelExtends.y, voxelExtends.z};
        if (vsg_store_create(e, &m_store) != VSG_OK) {
            std::cerr << "VoxelStreamingManager: invalid chunk extents" << std::endl;
            m_store = nullptr;
        }
    }
    ~VoxelStreamingManager() {
        if (m_store) vsg_store_destroy(m_store);
    }
    VoxelStreamingManager(const VoxelStreamingManager&) = delete;
    VoxelStreamingManager& operator=(const VoxelStreamingManager&) = delete;

    /* the calls below are synchronous: no auxiliary thread, no critical section */
    void startMultiThreading() {}
    void stopMultiThreading() {}
    void startAuxiliaryThread() {}
    void initializeCriticalSection() {}
    void deleteCriticalSection() {}

    void streamOut(VoxelScene& scene, const float3& cameraPos, float radius) {
        m_scene = &scene;
        streamOutFindBlocksOnGPU(vec3f(cameraPos.x, cameraPos.y, cameraPos.z), radius, false, false);
    }
    void streamIn(VoxelScene& scene, const float3& cameraPos, float radius) {
        m_scene = &scene;
        streamInCopyToGPUBuffer(vec3f(cameraPos.x, cameraPos.y, cameraPos.z), radius, false, false);
        streamInInsertToHashTable(false);
    }

    /* blocks at distance >= radius from sphereCenter leave the GPU */
    void streamOutFindBlocksOnGPU(const vec3f& sphereCenter, float radius, bool useParts, bool multiThreaded) {
        (void)useParts;
        (void)multiThreaded;
        if (!ready()) return;
        const float c[3] = {sphereCenter.x, sphereCenter.y, sphereCenter.z};
        uint32_t n = 0;
        if (vsg_stream_out(m_scene->handle(), m_store, c, radius, &n, nullptr) != VSG_OK)
            std::cerr << "[STREAM OUT] failed" << std::endl;
        m_out = n;
    }
    void streamOutCopyToChunkGrid(bool multiThreaded) { (void)multiThreaded; }

    void streamInCopyToGPUBuffer(const vec3f& sphereCenter, float radius, bool useParts, bool multiThreaded) {
        (void)useParts;
        (void)multiThreaded;
        m_inCenter = sphereCenter;
        m_inRadius = radius;
        m_inPending = true;
    }
    /* Takes the chunks chosen by the last streamInCopyToGPUBuffer, or, as
     * the reference's auxiliary thread would choose them, those around
     * posCamera_ within radius_ (voxelSG.cpp:528-551). */
    void streamInInsertToHashTable(bool multiThreaded) {
        (void)multiThreaded;
        if (!ready()) return;
        if (!m_inPending) {
            if (!(radius_ > 0.0f)) return;
            m_inCenter = posCamera_;
            m_inRadius = radius_;
        }
        m_inPending = false;
        const float c[3] = {m_inCenter.x, m_inCenter.y, m_inCenter.z};
        uint32_t n = 0, merged = 0;
        const int rc = vsg_stream_in(m_scene->handle(), m_store, c, m_inRadius, &n, &merged, nullptr);
        if (rc == VSG_ERR_TOO_LARGE)
            std::cerr << "[ERROR] Not enough free blocks in heap for stream-in" << std::endl;
        else if (rc != VSG_OK)
            std::cerr << "[STREAM IN] failed" << std::endl;
        m_in = n;
    }

    unsigned int getNumStreamedOut() const { return m_out; }
    unsigned int getNumStreamedIn() const { return m_in; }
    vsg_block_store* store() const { return m_store; }

    /* VoxelStreamingManager.cpp:836-903: file blocks given as the streaming
     * records (SDFBlockInfo array, SDFBlock array of 12-byte VoxelData). */
    void updateChunkGrid(const int* blockInfos, const int* blocks, unsigned int nSDFBlocks) {
        if (!m_store) return;
        if (vsg_store_add_records(m_store, m_params.voxelSize, reinterpret_cast<const int32_t*>(blockInfos),
                                  reinterpret_cast<const uint8_t*>(blocks), nSDFBlocks) != VSG_OK)
            std::cerr << "VoxelStreamingManager: updateChunkGrid failed" << std::endl;
    }
    /* VoxelStreamingManager.cpp:993-1140: the number of stored blocks a
     * stream-in around posCamera within radius takes (no chunk-grid bounds). */
    unsigned int streamInFindChunk(const vec3f& posCamera, float radius, bool useParts) {
        (void)useParts;
        uint64_t nb = 0;
        const float c[3] = {posCamera.x, posCamera.y, posCamera.z};
        if (!m_store || vsg_store_count(m_store, c, radius, &nb, nullptr) != VSG_OK) nb = 0;
        m_counter = (unsigned int)nb;
        return m_counter;
    }
    void clearSDFBlockCounter() { m_counter = 0; }
    unsigned int getSDFBlockCounter() const { return m_counter; }

    /* chunk helpers, VoxelStreamingManager.cpp:194-212, 905-991 */
    vec3i worldToChunks(const vec3f& posWorld) const {
        const float p[3] = {posWorld.x / m_ext.x, posWorld.y / m_ext.y, posWorld.z / m_ext.z};
        int c[3];
        for (int i = 0; i < 3; ++i) {
            const float s = p[i] > 0.0f ? 1.0f : (p[i] < 0.0f ? -1.0f : 0.0f);
            c[i] = static_cast<int>(p[i] + s * 0.5f);
        }
        return vec3i(c[0], c[1], c[2]);
    }
    bool isValidChunk(const vec3i& chunk) const {
        return chunk.x >= m_min.x && chunk.y >= m_min.y && chunk.z >= m_min.z && chunk.x < m_min.x + m_dims.x &&
               chunk.y < m_min.y + m_dims.y && chunk.z < m_min.z + m_dims.z;
    }
    unsigned int linearizeChunkPos(const vec3i& chunkPos) const {
        return (unsigned int)((chunkPos.z - m_min.z) * m_dims.x * m_dims.y + (chunkPos.y - m_min.y) * m_dims.x +
                              (chunkPos.x - m_min.x));
    }
    vec3i delinearizeChunkIndex(unsigned int idx) const {
        const unsigned int dx = (unsigned int)m_dims.x, dxy = (unsigned int)(m_dims.x * m_dims.y);
        return vec3i(m_min.x + (int)(idx % dx), m_min.y + (int)((idx % dxy) / dx), m_min.z + (int)(idx / dxy));
    }
    vec3i meterToNumberOfChunksCeil(float radius) const {
        return vec3i((int)std::ceil(radius / m_ext.x), (int)std::ceil(radius / m_ext.y), (int)std::ceil(radius / m_ext.z));
    }
    bool isChunkInSphere(const vec3i& chunk, const vec3f& center, float radius) const {
        const float wx = chunk.x * m_ext.x, wy = chunk.y * m_ext.y, wz = chunk.z * m_ext.z;
        const float ext = std::max(std::max(m_ext.x, m_ext.y), m_ext.z);
        const float r = 0.5f * ext * std::sqrt(3.0f);
        const float dx = wx - center.x, dy = wy - center.y, dz = wz - center.z;
        return std::sqrt(dx * dx + dy * dy + dz * dz) - r <= radius;
    }
    bool isInsideRadius(const float3& blockWorldCenter, const float3& cameraPos, float radius) const {
        const float dx = blockWorldCenter.x - cameraPos.x, dy = blockWorldCenter.y - cameraPos.y,
                    dz = blockWorldCenter.z - cameraPos.z;
        return dx * dx + dy * dy + dz * dz <= radius * radius;
    }
    float3 blockCoordToWorld(const int3& blockCoord) const {
        const float s = (float)SDF_BLOCK_SIZE * m_params.voxelSize;
        return make_float3(blockCoord.x * s, blockCoord.y * s, blockCoord.z * s);
    }

    /* runtime fields the reference's main loop sets (VoxelStreamingManager.h:287-292) */
    vec3f posCamera_;
    float radius_ = 0.0f;
    bool s_terminateThread = false;
    unsigned int m_frameNumber = 0;
    std::string m_outputDirectory;

private:
    bool ready() const {
        if (!m_store || !m_scene || !m_scene->isAllocated()) {
            std::cerr << "VoxelStreamingManager: scene or store not allocated" << std::endl;
            return false;
        }
        return true;
    }
    VoxelScene* m_scene;
    Params m_params;
    vsg_block_store* m_store = nullptr;
    vec3f m_inCenter;
    float m_inRadius = 0.0f;
    bool m_inPending = false;
    unsigned int m_out = 0, m_in = 0;
    unsigned int m_counter = 0;
    vec3f m_ext;
    vec3i m_dims, m_min;
};

/* CustomDepthMapGenerator (CustomDepthMapGenerator.h:15-165;
 * generateFromPointCloud, CustomDepthMapGenerator.cpp:81-222): point cloud
 * -> depth / point / normal / colour maps, computed on the GPU by
 * vsg_splat_points in the reference's order (the last point landing on a
 * pixel wins; a point's normal and colour are written only when it has
 * one; without normals the depth-map fallback).  Points, normals and colours
 * are any element types with .x/.y/.z (cv::Point3f) and operator[] (cv::Vec3b);
 * the maps come back as std::array elements.  Only the perspective
 * projection (PERSPECTIVE, CUSTOM_CAMERA) is implemented; ORTHOGRAPHIC
 * prints an error and returns empty maps. */
#include <array>

class CustomDepthMapGenerator {
public:
    struct CameraParams {
        float fx = 525.0f, fy = 525.0f, cx = 319.5f, cy = 239.5f;
        float nearPlane = 0.1f, farPlane = 10.0f;
        int width = 640, height = 480;
    };
    enum class ProjectionMethod { PERSPECTIVE, ORTHOGRAPHIC, CUSTOM_CAMERA };
    struct GeneratedDepthMap {
        std::vector<float> depthmap;                         // 0 = no point
        std::vector<std::array<float, 3>> pointmap;          // camera space, 0 = no point
        std::vector<std::array<float, 3>> normalmap;
        std::vector<std::array<unsigned char, 3>> colormap;
        int width = 0, height = 0;
    };

    void setCameraParams(const CameraParams& p) { m_cam = p; }
    void setCameraParams(float fx, float fy, float cx, float cy, float nearPlane, float farPlane, int width,
                         int height) {
        m_cam.fx = fx;
        m_cam.fy = fy;
        m_cam.cx = cx;
        m_cam.cy = cy;
        m_cam.nearPlane = nearPlane;
        m_cam.farPlane = farPlane;
        m_cam.width = width;
        m_cam.height = height;
    }
    const CameraParams& getCameraParams() const { return m_cam; }
    void setProjectionMethod(ProjectionMethod m) { m_method = m; }
    ProjectionMethod getProjectionMethod() const { return m_method; }

    template <class P, class N, class C>
    GeneratedDepthMap generateFromPointCloud(const std::vector<P>& points, const std::vector<N>& normals,
                                             const std::vector<C>& colors) {
        GeneratedDepthMap out;
        out.width = m_cam.width;
        out.height = m_cam.height;
        if (m_method == ProjectionMethod::ORTHOGRAPHIC) {
            std::cerr << "CustomDepthMapGenerator: only the perspective projection is implemented" << std::endl;
            return out;
        }
        const size_t npx = (size_t)m_cam.width * (size_t)m_cam.height;
        std::vector<float> hp(3 * points.size()), hn(3 * normals.size());
        std::vector<unsigned char> hc(3 * colors.size());
        for (size_t i = 0; i < points.size(); ++i) {
            hp[3 * i] = points[i].x;
            hp[3 * i + 1] = points[i].y;
            hp[3 * i + 2] = points[i].z;
        }
        for (size_t i = 0; i < normals.size(); ++i) {
            hn[3 * i] = normals[i].x;
            hn[3 * i + 1] = normals[i].y;
            hn[3 * i + 2] = normals[i].z;
        }
        for (size_t i = 0; i < colors.size(); ++i)
            for (int k = 0; k < 3; ++k) hc[3 * i + k] = (unsigned char)colors[i][k];
        float *dp = nullptr, *dn = nullptr, *dd = nullptr, *dpm = nullptr, *dnm = nullptr;
        unsigned char *dc = nullptr, *dcm = nullptr;
        bool ok = cudaMalloc(&dp, hp.size() * 4 + 4) == cudaSuccess &&
                  cudaMalloc(&dn, hn.size() * 4 + 4) == cudaSuccess &&
                  cudaMalloc(&dc, hc.size() + 4) == cudaSuccess && cudaMalloc(&dd, npx * 4) == cudaSuccess &&
                  cudaMalloc(&dpm, npx * 12) == cudaSuccess && cudaMalloc(&dnm, npx * 12) == cudaSuccess &&
                  cudaMalloc(&dcm, npx * 3) == cudaSuccess;
        if (ok)
            ok = cudaMemcpy(dp, hp.data(), hp.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
                 cudaMemcpy(dn, hn.data(), hn.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
                 cudaMemcpy(dc, hc.data(), hc.size(), cudaMemcpyHostToDevice) == cudaSuccess;
        int64_t nvalid = 0;
        if (ok)
            ok = vsg_splat_points(dp, (int64_t)points.size(), dn, (int64_t)normals.size(), dc, (int64_t)colors.size(),
                                  m_cam.width, m_cam.height, m_cam.fx, m_cam.fy, m_cam.cx, m_cam.cy, 0.0f,
                                  std::numeric_limits<float>::infinity(), VSG_SPLAT_LAST, dd, dpm, dnm, dcm,
                                  &nvalid, nullptr) == VSG_OK;
        if (ok) {
            out.depthmap.resize(npx);
            out.pointmap.resize(npx);
            out.normalmap.resize(npx);
            out.colormap.resize(npx);
            ok = cudaMemcpy(out.depthmap.data(), dd, npx * 4, cudaMemcpyDeviceToHost) == cudaSuccess &&
                 cudaMemcpy(out.pointmap.data(), dpm, npx * 12, cudaMemcpyDeviceToHost) == cudaSuccess &&
                 cudaMemcpy(out.normalmap.data(), dnm, npx * 12, cudaMemcpyDeviceToHost) == cudaSuccess &&
                 cudaMemcpy(out.colormap.data(), dcm, npx * 3, cudaMemcpyDeviceToHost) == cudaSuccess;
        }
        cudaFree(dp);
        cudaFree(dn);
        cudaFree(dc);
        cudaFree(dd);
        cudaFree(dpm);
        cudaFree(dnm);
        cudaFree(dcm);
        if (!ok) {
            std::cerr << "CustomDepthMapGenerator: point cloud splat failed" << std::endl;
            out.depthmap.clear();
            out.pointmap.clear();
            out.normalmap.clear();
            out.colormap.clear();
        }
        return out;
    }

private:
    CameraParams m_cam;
    ProjectionMethod m_method = ProjectionMethod::PERSPECTIVE;
};
