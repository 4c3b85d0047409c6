// Host voxelizer types (crates/cfd/src/voxel.rs restated in C++).
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace lbm {

struct Surface {  // voxel.rs:24-29
    std::vector<std::array<double, 3>> verts;
    std::vector<std::array<uint32_t, 3>> tris;
};

struct GridSpec {  // voxel.rs:49-66: points origin + h * (i, j, k)
    std::array<double, 3> origin{};
    double h = 1.0;
    std::array<size_t, 3> dims{};
};

struct WallCell {  // voxel.rs:328-335
    uint32_t cell = 0;
    uint32_t mask = 0;
    std::array<float, 27> q{};
};

struct StaticVoxels {  // voxel.rs:337-344
    std::vector<uint32_t> solid;
    std::vector<WallCell> walls;
    std::array<size_t, 3> lo{}, hi{};
};

struct SpinVoxels {  // voxel.rs:492-505 (the diagnostic bins are left out)
    std::array<double, 3> occ_lo{};
    double occ_h = 0.125;
    std::array<size_t, 3> occ_dims{};
    std::vector<uint32_t> occ_bits;
    std::vector<std::array<float, 12>> tris;  // v0, e1, e2 (body frame), each padded to 4
    double radius = 0;
    double axial[2] = {0, 0};
};

std::vector<uint8_t> inside_grid(const Surface &s, const GridSpec &g);
Surface subdivide(const Surface &s, double max_edge);
SpinVoxels voxelize_spin(const Surface &s, std::array<double, 3> axis, double h);
bool seg_tri(const double o[3], const double d[3], const double t0[3], const double t1[3], const double t2[3], double *t);
StaticVoxels voxelize_static(const Surface &s, std::array<size_t, 3> dims, int lattice);
const std::vector<std::array<int, 3>> &dirs19();
const std::vector<std::array<int, 3>> &dirs27();

// Failure of the GPU voxelizer: code 1 internal, 2 out of device memory, 3 CUDA error
struct VoxelError : std::runtime_error {
    int code;
    VoxelError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};
// voxelize_static on the current CUDA device: the same solid cells and wall
// links, bit for bit
StaticVoxels voxelize_static_gpu(const Surface &s, std::array<size_t, 3> dims, int lattice);

}  // namespace lbm
