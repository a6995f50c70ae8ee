// vpt_sparse.h - sparse (NanoVDB-compatible) volumes: host-side construction of the SparseView the
// tracer reads (vpt_params.h).
//
// Two ways in, one layout out:
//  * parse_nanovdb: a NanoVDB float grid buffer (version 32, as written by nanovdb::io or built by
//    GridBuilder), the reference's `.nvdb` path (CloudData::loadFromNvdbFile, CloudData.cpp:1360-1365);
//  * build_sparse_from_dense: the dense -> sparse conversion of CloudData::getSparseDensityField
//    (CloudData.cpp:1385-1407), which runs nanovdb::GridBuilder with background 0 over the index box
//    [0, n-1]: voxels != 0 become active leaf values, a leaf whose 512 voxels are all active and
//    equal becomes an active lower-node tile, a lower node whose 4096 slots are such tiles of one
//    value becomes an active upper tile, and so on (GridBuilder.h:251-340); node bounding boxes are
//    the active-value boxes of GridStats (GridStats.h:620-700).
// Both produce the brick table (one entry per 8^3 brick over the root box rounded out to 128-voxel
// node boundaries), the tile list with each tile's node box, the per-leaf LeafData::mBBoxMin and
// the leaf value/mask pools on the device.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include "vpt_params.h"

namespace vpt {

struct SparseHost {
    float mat[9] = {0}, inv_mat[9] = {0}, vec[3] = {0};
    double world_min[3] = {0}, world_max[3] = {0};  // GridData::mWorldBBox
    double voxel_size[3] = {0};                      // GridData::mVoxelSize
    int root_min[3] = {0}, root_max[3] = {-1, -1, -1};
    float background = 0.0f;
    int tbl_origin[3] = {0}, tbl_dim[3] = {0};
    std::vector<uint32_t> table;
    std::vector<SparseTile> tiles;
    struct RootTile {
        int origin[3];
        int child;
        float value;
        int active;
    };
    std::vector<RootTile> root_tiles;  // in the order of the root's tile table
    std::vector<int> leaf_bbox_min;  // 3 per leaf
    std::vector<uint64_t> leaf_src;  // per leaf: byte offset of the LeafNode in the source buffer, or the
                                     // linear index of the source brick (dense build)
    size_t leaf_count() const { return leaf_src.size(); }
};

// Device storage of a sparse volume (owned by the context).
struct SparseDevice {
    uint32_t* table = nullptr;
    SparseTile* tiles = nullptr;
    int* leaf_bbox_min = nullptr;
    float* values = nullptr;
    unsigned short* values_h = nullptr;
    uint32_t* masks = nullptr;
    size_t leaves = 0;
    size_t bytes = 0;
    void release();
};

// Parses a NanoVDB float grid in host memory into `out` (no device work).  Returns false with a
// message for buffers that are not a version-32 float grid.
bool parse_nanovdb(const uint8_t* buf, size_t bytes, SparseHost& out, std::string& err);

// Uploads `h` and gathers the leaf values (optionally as fp16) and masks from the NanoVDB buffer
// `dev_buf` (device memory, the same bytes that parse_nanovdb read).
cudaError_t upload_sparse_from_nanovdb(const SparseHost& h, const uint8_t* dev_buf, bool fp16, SparseDevice& d,
                                       cudaStream_t s);

// Dense grid (device, x fastest, nx*ny*nz floats, values as the tracer should read them) -> sparse
// volume with the voxel size `dx` and world origin `origin` (GridBuilder::getHandle(dx, origin)).
cudaError_t build_sparse_from_dense(const float* dense, int nx, int ny, int nz, double dx, const double origin[3],
                                    bool fp16, SparseHost& h, SparseDevice& d, cudaStream_t s, std::string& err);

// The tracer's view of a built volume.
SparseView make_sparse_view(const SparseHost& h, const SparseDevice& d, int lowest_level);

}  // namespace vpt
