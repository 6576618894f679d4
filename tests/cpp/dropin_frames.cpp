// Drive the fusion path through the C++ drop-in classes the way the
// reference's main loop does (voxelSG.cpp:392-618): configure the knobs,
// build a VoxelScene, and per frame upload the maps, integrateFromScanData,
// construct a RayCastRender, render at the frame's pose from a device
// matrix, download the depth.  After the frames it extracts the surface with
// the marching-cubes launchers (MarchingCubes.h:34-58) and streams blocks
// out to host memory and back with VoxelStreamingManager, then renders the
// last pose again.  The last frame's render and surface points go to PLY
// files.  Built with -DUSE_NORMAL_DIR_ALLOC it runs the reference's
// normal-direction allocation (Method 2).  Test harness: frames come from
// binary files written by the Python test, depths are written back for
// comparison.
//
//   dropin_frames DIR NFRAMES W H FX FY CX CY VOXEL TRUNC SLOTS BLOCKS MIND MAXD
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "voxelsg_b200.hpp"

static bool read_file(const std::string& path, void* dst, size_t bytes) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    const size_t got = std::fread(dst, 1, bytes, f);
    std::fclose(f);
    return got == bytes;
}

static bool write_file(const std::string& path, const void* src, size_t bytes) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const size_t put = std::fwrite(src, 1, bytes, f);
    std::fclose(f);
    return put == bytes;
}

int main(int argc, char** argv) {
    if (argc != 15) {
        std::fprintf(stderr, "usage: %s DIR NFRAMES W H FX FY CX CY VOXEL TRUNC SLOTS BLOCKS MIND MAXD\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const int nframes = std::atoi(argv[2]), W = std::atoi(argv[3]), H = std::atoi(argv[4]);
    const float fx = std::atof(argv[5]), fy = std::atof(argv[6]), cx = std::atof(argv[7]), cy = std::atof(argv[8]);
    GlobalParamsConfig& g = GlobalParamsConfig::get();
    g.g_SDFVoxelSize = std::atof(argv[9]);
    g.g_SDFTruncation = std::atof(argv[10]);
    g.g_hashNumSlots = g.g_hashNumBuckets = (unsigned)std::atoi(argv[11]);
    g.g_hashNumSDFBlocks = (unsigned)std::atoi(argv[12]);
    const float minD = std::atof(argv[13]), maxD = std::atof(argv[14]);
    g.initialize();
    Params params(g);
    VoxelScene scene(params);
    if (!scene.isAllocated()) return 3;
    const size_t n = (size_t)W * H;
    std::vector<float> pm(3 * n), nm(3 * n), depth(n);
    std::vector<unsigned char> rgb(3 * n);
    float3 *d_pm = nullptr, *d_nm = nullptr;
    uchar3* d_rgb = nullptr;
    float* d_T = nullptr;
    cudaMalloc(&d_pm, n * sizeof(float3));
    cudaMalloc(&d_nm, n * sizeof(float3));
    cudaMalloc(&d_rgb, n * sizeof(uchar3));
    cudaMalloc(&d_T, 16 * sizeof(float));
    for (int i = 0; i < nframes; ++i) {
        vsg::Mat4f T;
        const std::string id = std::to_string(i);
        if (!read_file(dir + "/pm_" + id + ".bin", pm.data(), pm.size() * 4) ||
            !read_file(dir + "/rgb_" + id + ".bin", rgb.data(), rgb.size()) ||
            !read_file(dir + "/nm_" + id + ".bin", nm.data(), nm.size() * 4) ||
            !read_file(dir + "/pose_" + id + ".bin", T.m, sizeof(T.m)))
            return 4;
        cudaMemcpy(d_pm, pm.data(), n * sizeof(float3), cudaMemcpyHostToDevice);
        cudaMemcpy(d_nm, nm.data(), n * sizeof(float3), cudaMemcpyHostToDevice);
        cudaMemcpy(d_rgb, rgb.data(), n * sizeof(uchar3), cudaMemcpyHostToDevice);
        scene.integrateFromScanData(d_pm, d_rgb, d_nm, W, H, g.g_SDFTruncation, T, fx, fy, cx, cy);
        RayCastRender renderer;  // the reference builds one per frame (voxelSG.cpp:578)
        if (!renderer.initialize(W, H)) return 5;
        const float3 cam = make_float3(T.at<float>(0, 3), T.at<float>(1, 3), T.at<float>(2, 3));
        cudaMemcpy(d_T, T.m, sizeof(T.m), cudaMemcpyHostToDevice);
        renderer.render(&scene, cam, d_T, fx, fy, cx, cy, minD, maxD);
        renderer.downloadDepthFloat(depth.data());
        if (!write_file(dir + "/depth_" + id + ".bin", depth.data(), n * 4)) return 6;
        if (i == nframes - 1) {
            // the exporters the reference's main loop calls (voxelSG.cpp:656-673)
            if (!renderer.savePointCloudPLY(dir + "/cloud.ply")) return 8;
            std::printf("surface_points=%d\n", renderer.extractSurfacePoints(&scene, -0.1f, 0.1f, 1));
            if (!renderer.saveExtractedSurfacePointsPLY(dir + "/surface.ply")) return 9;
        }
    }
    std::printf("frames=%u free=%u\n", scene.getNumIntegratedFrames(), scene.getHeapFreeCount());
    // marching cubes as the reference's launchers are called
    MarchingCubesParams mcParams;
    mcParams.voxelSize = g.g_SDFVoxelSize;
    MarchingCubesOutput mcOut;
    allocateMarchingCubesOutput(mcOut, (int)g.g_marchingCubesMaxNumTriangles);
    runMarchingCubesCUDA(scene.getHashData(), scene.getParams(), mcParams, mcOut);
    std::printf("triangles=%d\n", copyMarchingCubesTriangleCount(mcOut));
    freeMarchingCubesOutput(mcOut);
    scene.compactifyHashEntries();
    scene.printStats();
    if (!scene.saveToMesh(dir + "/mesh.ply")) return 10;
    // stream far blocks out, then everything back in, and render the last pose again
    VoxelStreamingManager streaming(scene, params, vec3f(0.1f, 0.1f, 0.1f), vec3i(513, 513, 513),
                                    vec3i(-256, -256, -256), 2000, false);
    streaming.streamOutFindBlocksOnGPU(vec3f(0.0f, 0.1f, 0.0f), 0.25f, false, false);
    streaming.streamOutCopyToChunkGrid(false);
    std::printf("streamed_out=%u free=%u\n", streaming.getNumStreamedOut(), scene.getHeapFreeCount());
    // stream-in as the reference's main loop drives it: the sphere in
    // posCamera_ / radius_, then the insert (voxelSG.cpp:528-551)
    std::printf("found=%u\n", streaming.streamInFindChunk(vec3f(0.0f, 0.1f, 0.0f), 100.0f, false));
    streaming.posCamera_ = vec3f(0.0f, 0.1f, 0.0f);
    streaming.radius_ = 100.0f;
    streaming.streamInInsertToHashTable(true);
    std::printf("streamed_in=%u free=%u\n", streaming.getNumStreamedIn(), scene.getHeapFreeCount());
    {
        vsg::Mat4f T;
        if (!read_file(dir + "/pose_" + std::to_string(nframes - 1) + ".bin", T.m, sizeof(T.m))) return 4;
        RayCastRender renderer;
        if (!renderer.initialize(W, H)) return 5;
        const float3 cam = make_float3(T.at<float>(0, 3), T.at<float>(1, 3), T.at<float>(2, 3));
        cudaMemcpy(d_T, T.m, sizeof(T.m), cudaMemcpyHostToDevice);
        renderer.render(&scene, cam, d_T, fx, fy, cx, cy, minD, maxD);
        renderer.downloadDepthFloat(depth.data());
        if (!write_file(dir + "/depth_after_stream.bin", depth.data(), n * 4)) return 6;
    }
    cudaFree(d_pm);
    cudaFree(d_nm);
    cudaFree(d_rgb);
    cudaFree(d_T);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 7;
}
