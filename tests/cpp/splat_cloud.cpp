// Run CustomDepthMapGenerator (the C++ drop-in) on a point cloud read from
// binary files and write its four maps back, for comparison with the
// Python binding of vsg_splat_points.
//
//   splat_cloud DIR N_POINTS N_NORMALS N_COLORS W H FX FY CX CY
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "voxelsg_b200.hpp"

struct P3 {
    float x, y, z;
};

static bool read_file(const std::string& path, void* dst, size_t bytes) {
    if (bytes == 0) return true;
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
    if (argc != 11) {
        std::fprintf(stderr, "usage: %s DIR N_POINTS N_NORMALS N_COLORS W H FX FY CX CY\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const size_t np = std::strtoull(argv[2], nullptr, 10), nn = std::strtoull(argv[3], nullptr, 10),
                 nc = std::strtoull(argv[4], nullptr, 10);
    const int W = std::atoi(argv[5]), H = std::atoi(argv[6]);
    std::vector<P3> pts(np), nrm(nn);
    std::vector<std::array<unsigned char, 3>> col(nc);
    if (!read_file(dir + "/points.bin", pts.data(), np * 12) || !read_file(dir + "/normals.bin", nrm.data(), nn * 12) ||
        !read_file(dir + "/colors.bin", col.data(), nc * 3))
        return 3;
    CustomDepthMapGenerator gen;
    gen.setCameraParams((float)std::atof(argv[7]), (float)std::atof(argv[8]), (float)std::atof(argv[9]),
                        (float)std::atof(argv[10]), 0.1f, 10.0f, W, H);
    const CustomDepthMapGenerator::GeneratedDepthMap m = gen.generateFromPointCloud(pts, nrm, col);
    const size_t n = (size_t)W * H;
    if (m.depthmap.size() != n) return 4;
    if (!write_file(dir + "/depth.bin", m.depthmap.data(), n * 4) ||
        !write_file(dir + "/pointmap.bin", m.pointmap.data(), n * 12) ||
        !write_file(dir + "/normalmap.bin", m.normalmap.data(), n * 12) ||
        !write_file(dir + "/colormap.bin", m.colormap.data(), n * 3))
        return 5;
    return 0;
}
