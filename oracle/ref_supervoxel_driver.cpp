// ref_supervoxel_driver.cpp - C entry points over the reference's own supervoxel grid builders
// (TEST INFRASTRUCTURE ONLY).  SuperVoxelGrid.cpp and DensityField.cpp are compiled unmodified from the
// reference tree against oracle/ref_cpp_shim (oracle/ref_build.py); the grids are read back from the
// data the builders upload to their (shimmed) textures.
#include <stdint.h>
#include <string.h>

#include "DensityField.hpp"
#include "SuperVoxelGrid.hpp"

namespace {
DensityFieldPtr field_of(const float* raw, int nx, int ny, int nz) {
    const size_t n = (size_t)nx * ny * nz;
    auto* data = new float[n];  // owned by the DensityField (DensityField.cpp:46-50)
    memcpy(data, raw, n * sizeof(float));
    return std::make_shared<DensityField>(n, data);
}

GridInterpolationType interp_of(int interp) {
    return interp == 0 ? GridInterpolationType::NEAREST
                       : (interp == 1 ? GridInterpolationType::STOCHASTIC : GridInterpolationType::TRILINEAR);
}

void copy_out(const sgl::vk::TexturePtr& tex, void* out, size_t bytes) {
    const auto& b = tex->getImage()->bytes;
    memcpy(out, b.data(), std::min(bytes, b.size()));
}
}  // namespace

extern "C" {

// SuperVoxelGridResidualRatioTracking on the raw grid (normalised by DensityField::getDataFloatAtNorm):
// (mu_c, mu_r_bar) per supervoxel (after setExtinction) and the occupancy; dims[0..3] = grid size x, y,
// z and the supervoxel size.  Returns 0 on success.
int ref_supervoxel_rrt(const float* raw, int nx, int ny, int nz, int sv, int interp, int clamp_to_zero_border,
                       float extinction, float* out_pairs, uint8_t* out_occ, int* dims) {
    sgl::vk::Device device;
    SuperVoxelGridResidualRatioTracking grid(&device, nx, ny, nz, field_of(raw, nx, ny, nz), sv,
                                             clamp_to_zero_border != 0, interp_of(interp));
    grid.setExtinction(extinction);
    const glm::ivec3 g = grid.getSuperVoxelGridSize();
    dims[0] = g.x;
    dims[1] = g.y;
    dims[2] = g.z;
    dims[3] = grid.getSuperVoxelSize().x;
    const size_t count = (size_t)g.x * g.y * g.z;
    if (out_pairs) copy_out(grid.getSuperVoxelGridTexture(), out_pairs, count * 2 * sizeof(float));
    if (out_occ) copy_out(grid.getSuperVoxelGridOccupancyTexture(), out_occ, count);
    return 0;
}

// SuperVoxelGridDecompositionTracking: (min, max) normalised density per supervoxel and the occupancy.
int ref_supervoxel_decomposition(const float* raw, int nx, int ny, int nz, int sv, int interp,
                                 int clamp_to_zero_border, float* out_minmax, uint8_t* out_occ, int* dims) {
    sgl::vk::Device device;
    SuperVoxelGridDecompositionTracking grid(&device, nx, ny, nz, field_of(raw, nx, ny, nz), sv,
                                             clamp_to_zero_border != 0, interp_of(interp));
    const glm::ivec3 g = grid.getSuperVoxelGridSize();
    dims[0] = g.x;
    dims[1] = g.y;
    dims[2] = g.z;
    dims[3] = grid.getSuperVoxelSize().x;
    const size_t count = (size_t)g.x * g.y * g.z;
    if (out_minmax) copy_out(grid.getSuperVoxelGridTexture(), out_minmax, count * 2 * sizeof(float));
    if (out_occ) copy_out(grid.getSuperVoxelGridOccupancyTexture(), out_occ, count);
    return 0;
}

}  // extern "C"
