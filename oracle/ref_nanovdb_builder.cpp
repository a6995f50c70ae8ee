// ref_nanovdb_builder.cpp - TEST INFRASTRUCTURE ONLY.  Compiled by oracle/ref_build.py against the
// reference's vendored NanoVDB headers (src/nanovdb/NanoVDB.h, src/nanovdb/util/GridBuilder.h); the
// output library lives in oracle/_ref/.  It builds a NanoVDB float grid from a dense grid exactly as
// CloudData::getSparseDensityField does (src/CloudData.cpp:1385-1407): GridBuilder with background
// 0, one functor value per voxel x + (y + z*ny)*nx over the index box [0, n-1], voxel size dx,
// origin = the dense box minimum, GridClass::FogVolume.
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include <nanovdb/NanoVDB.h>
#include <nanovdb/util/GridBuilder.h>

extern "C" {

// Returns the grid buffer (malloc'ed, free with refvdb_free) and its size in bytes.
int refvdb_build_from_dense(const float* dense, int nx, int ny, int nz, double dx, double ox, double oy, double oz,
                            uint8_t** out, uint64_t* out_size) {
    nanovdb::GridBuilder<float> builder(0.0f);
    auto op = [&](const nanovdb::Coord& ijk) -> float {
        auto x = uint32_t(ijk.x());
        auto y = uint32_t(ijk.y());
        auto z = uint32_t(ijk.z());
        return dense[x + (y + size_t(z) * uint32_t(ny)) * uint32_t(nx)];
    };
    builder(op, nanovdb::CoordBBox(nanovdb::Coord(0), nanovdb::Coord(nx - 1, ny - 1, nz - 1)));
    auto handle = builder.getHandle<>(dx, nanovdb::Vec3d(ox, oy, oz), "density", nanovdb::GridClass::FogVolume);
    const uint64_t size = handle.size();
    auto* buf = static_cast<uint8_t*>(std::malloc(size));
    if (!buf) return 1;
    std::memcpy(buf, handle.data(), size);
    *out = buf;
    *out_size = size;
    return 0;
}

void refvdb_free(uint8_t* p) { std::free(p); }

// World bounding box of the grid (GridData::mWorldBBox) and its index bounding box, as
// CloudData::computeSparseGridMetadata reads them (src/CloudData.cpp:1289-1330).
int refvdb_grid_info(const uint8_t* buf, double world_bbox[6], int32_t index_bbox[6], double voxel_size[3]) {
    const auto* grid = reinterpret_cast<const nanovdb::NanoGrid<float>*>(buf);
    if (!grid->isValid()) return 1;
    auto wb = grid->worldBBox();
    auto ib = grid->indexBBox();
    for (int i = 0; i < 3; i++) {
        world_bbox[i] = wb.min()[i];
        world_bbox[3 + i] = wb.max()[i];
        index_bbox[i] = ib.min()[i];
        index_bbox[3 + i] = ib.max()[i];
        voxel_size[i] = grid->voxelSize()[i];
    }
    return 0;
}

}  // extern "C"
