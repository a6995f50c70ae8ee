// vpt_sparse.cu - construction of sparse volumes (see vpt_sparse.h).
//
// NanoVDB layout read here (version 32, float grids; offsets as in the NanoVDB headers and
// PNanoVDB.glsl:712-1171): GridData 672 B (map at 296: mMatF, mInvMatF, mVecF; world bbox at 560;
// grid type at 636), TreeData 64 B (root offset at 24), RootData 64 B (bbox at 0/12, tile count at 24,
// background at 28) followed by 32-byte tiles (key, child offset, state, value), upper nodes (value
// mask at 32, child mask at 4128, 8-byte table at 8256), lower nodes (masks at 32/544, table at
// 1088), leaves (mBBoxMin at 0, value mask at 16, 512 floats at 96).  Child offsets are relative to
// the parent node.
#include "vpt_sparse.h"

#include <cuda_fp16.h>
#include <math.h>
#include <string.h>
#include <algorithm>
#include <climits>
#include <map>
#include <tuple>
#include "vpt_kernels.h"

namespace vpt {

namespace {

constexpr uint64_t kNanoMagic = 0x304244566f6e614eULL;  // "NanoVDB0"
constexpr size_t kGridSize = 672, kTreeSize = 64, kRootSize = 64, kRootTileSize = 32;
constexpr size_t kUpperValueMask = 32, kUpperChildMask = 4128, kUpperTable = 8256, kUpperSize = 270400;
constexpr size_t kLowerValueMask = 32, kLowerChildMask = 544, kLowerTable = 1088, kLowerSize = 33856;
constexpr size_t kLeafValueMask = 16, kLeafValues = 96, kLeafSize = 2144;

template <class T>
T rd(const uint8_t* b, size_t off) {
    T v;
    memcpy(&v, b + off, sizeof(T));
    return v;
}
bool bit(const uint8_t* b, size_t mask_off, uint32_t n) {
    return (rd<uint32_t>(b, mask_off + 4 * (n >> 5)) >> (n & 31u)) & 1u;
}

struct TileKey {
    uint32_t value_bits;
    int active, level;
    int box[6];
    bool operator<(const TileKey& o) const {
        return std::tie(value_bits, active, level, box[0], box[1], box[2], box[3], box[4], box[5]) <
               std::tie(o.value_bits, o.active, o.level, o.box[0], o.box[1], o.box[2], o.box[3], o.box[4], o.box[5]);
    }
};

struct Assembler {
    SparseHost& h;
    std::map<TileKey, uint32_t> tile_index;

    explicit Assembler(SparseHost& host) : h(host) {}

    // Table over the root box, rounded out to 128-voxel (lower node) boundaries, so that every cell
    // the HDDA can visit next to the active region reports its node exactly.
    bool init_table(std::string& err) {
        for (int a = 0; a < 3; a++) {
            if (h.root_max[a] < h.root_min[a]) {
                h.tbl_dim[0] = h.tbl_dim[1] = h.tbl_dim[2] = 0;
                h.table.clear();
                return true;
            }
        }
        size_t n = 1;
        for (int a = 0; a < 3; a++) {
            const long long lo = (long long)(h.root_min[a] >> 7) << 7;
            const long long hi = ((long long)(h.root_max[a] >> 7) << 7) + 128;
            h.tbl_origin[a] = (int)lo;
            h.tbl_dim[a] = (int)((hi - lo) >> 3);
            n *= (size_t)h.tbl_dim[a];
        }
        if (n > (size_t(1) << 31)) {
            err = "sparse grid bounding box too large for the brick table";
            return false;
        }
        SparseTile bg{};
        bg.value = h.background;
        bg.level = 4;
        h.table.assign(n, tile(bg));
        return true;
    }

    uint32_t tile(const SparseTile& t) {
        TileKey k;
        memcpy(&k.value_bits, &t.value, 4);
        k.active = t.active;
        k.level = t.level;
        for (int i = 0; i < 6; i++) k.box[i] = t.box[i];
        auto it = tile_index.find(k);
        if (it != tile_index.end()) return it->second;
        const uint32_t entry = kSparseTileBit | (uint32_t)h.tiles.size();
        h.tiles.push_back(t);
        tile_index.emplace(k, entry);
        return entry;
    }

    // Sets every brick of the cube [o, o + size) that lies in the table.
    void fill(const long long o[3], long long size, uint32_t entry) {
        long long b0[3], b1[3];
        for (int a = 0; a < 3; a++) {
            b0[a] = std::max<long long>((o[a] - h.tbl_origin[a]) >> 3, 0);
            b1[a] = std::min<long long>((o[a] + size - h.tbl_origin[a] + 7) >> 3, h.tbl_dim[a]);
            if (b1[a] <= b0[a]) return;
        }
        for (long long z = b0[2]; z < b1[2]; z++)
            for (long long y = b0[1]; y < b1[1]; y++)
                for (long long x = b0[0]; x < b1[0]; x++)
                    h.table[((size_t)z * h.tbl_dim[1] + (size_t)y) * h.tbl_dim[0] + (size_t)x] = entry;
    }

    bool intersects(const long long o[3], long long size) const {
        for (int a = 0; a < 3; a++) {
            const long long t0 = h.tbl_origin[a], t1 = (long long)h.tbl_origin[a] + 8LL * h.tbl_dim[a];
            if (o[a] + size <= t0 || o[a] >= t1) return false;
        }
        return true;
    }
};

SparseTile make_tile(float value, bool active, int level, const int* box) {
    SparseTile t{};
    t.value = value;
    t.active = active ? 1 : 0;
    t.level = level;
    for (int i = 0; i < 6; i++) t.box[i] = box ? box[i] : 0;
    return t;
}

}  // namespace

void SparseDevice::release() {
    cudaFree(table);
    cudaFree(tiles);
    cudaFree(leaf_bbox_min);
    cudaFree(values);
    cudaFree(values_h);
    cudaFree(masks);
    *this = SparseDevice();
}

bool parse_nanovdb(const uint8_t* b, size_t bytes, SparseHost& h, std::string& err) {
    h = SparseHost();
    if (bytes < kGridSize + kTreeSize + kRootSize || rd<uint64_t>(b, 0) != kNanoMagic) {
        err = "not a NanoVDB grid buffer";
        return false;
    }
    const uint32_t version = rd<uint32_t>(b, 16);
    if ((version >> 21) != 32u) {
        err = "unsupported NanoVDB version (major 32 expected)";
        return false;
    }
    if (rd<uint32_t>(b, 636) != 1u) {
        err = "unsupported NanoVDB grid type (float grids only)";
        return false;
    }
    for (int i = 0; i < 9; i++) {
        h.mat[i] = rd<float>(b, 296 + 4 * i);
        h.inv_mat[i] = rd<float>(b, 296 + 36 + 4 * i);
    }
    for (int i = 0; i < 3; i++) h.vec[i] = rd<float>(b, 296 + 72 + 4 * i);
    for (int i = 0; i < 3; i++) {
        h.world_min[i] = rd<double>(b, 560 + 8 * i);
        h.world_max[i] = rd<double>(b, 584 + 8 * i);
        h.voxel_size[i] = rd<double>(b, 608 + 8 * i);
    }
    const size_t tree = kGridSize;
    const size_t root = tree + rd<uint64_t>(b, tree + 24);
    if (root + kRootSize > bytes) {
        err = "truncated NanoVDB buffer (root)";
        return false;
    }
    for (int i = 0; i < 3; i++) {
        h.root_min[i] = rd<int32_t>(b, root + 4 * i);
        h.root_max[i] = rd<int32_t>(b, root + 12 + 4 * i);
    }
    const uint32_t tile_count = rd<uint32_t>(b, root + 24);
    h.background = rd<float>(b, root + 28);
    if (root + kRootSize + (size_t)tile_count * kRootTileSize > bytes) {
        err = "truncated NanoVDB buffer (root tiles)";
        return false;
    }
    Assembler as(h);
    if (!as.init_table(err)) return false;
    if (h.table.empty()) return true;
    int root_box[6];
    for (int i = 0; i < 3; i++) {
        root_box[i] = h.root_min[i];
        root_box[3 + i] = h.root_max[i];
    }
    for (uint32_t t = 0; t < tile_count; t++) {
        const size_t tile = root + kRootSize + (size_t)t * kRootTileSize;
        const uint64_t key = rd<uint64_t>(b, tile);
        const int64_t child = rd<int64_t>(b, tile + 8);
        long long o[3] = {(long long)(int32_t)((uint32_t)((key >> 42) & 0x1FFFFFu) << 12),
                          (long long)(int32_t)((uint32_t)((key >> 21) & 0x1FFFFFu) << 12),
                          (long long)(int32_t)((uint32_t)(key & 0x1FFFFFu) << 12)};
        h.root_tiles.push_back({{(int)o[0], (int)o[1], (int)o[2]}, child != 0 ? 1 : 0, rd<float>(b, tile + 20),
                                rd<uint32_t>(b, tile + 16) != 0u ? 1 : 0});
        if (!as.intersects(o, 4096)) continue;
        if (child == 0) {
            as.fill(o, 4096, as.tile(make_tile(rd<float>(b, tile + 20), rd<uint32_t>(b, tile + 16) != 0u, 3, root_box)));
            continue;
        }
        const size_t upper = root + (size_t)child;
        if (upper + kUpperSize > bytes) {
            err = "truncated NanoVDB buffer (upper node)";
            return false;
        }
        int upper_box[6];
        for (int i = 0; i < 6; i++) upper_box[i] = rd<int32_t>(b, upper + 4 * i);
        for (uint32_t n = 0; n < 32768u; n++) {
            long long uo[3] = {o[0] + (long long)(n >> 10) * 128, o[1] + (long long)((n >> 5) & 31u) * 128,
                               o[2] + (long long)(n & 31u) * 128};
            if (!as.intersects(uo, 128)) continue;
            if (!bit(b, upper + kUpperChildMask, n)) {
                as.fill(uo, 128, as.tile(make_tile(rd<float>(b, upper + kUpperTable + 8 * n),
                                                   bit(b, upper + kUpperValueMask, n), 2, upper_box)));
                continue;
            }
            const size_t lower = upper + (size_t)rd<int64_t>(b, upper + kUpperTable + 8 * n);
            if (lower + kLowerSize > bytes) {
                err = "truncated NanoVDB buffer (lower node)";
                return false;
            }
            int lower_box[6];
            for (int i = 0; i < 6; i++) lower_box[i] = rd<int32_t>(b, lower + 4 * i);
            for (uint32_t m = 0; m < 4096u; m++) {
                long long lo[3] = {uo[0] + (long long)(m >> 8) * 8, uo[1] + (long long)((m >> 4) & 15u) * 8,
                                   uo[2] + (long long)(m & 15u) * 8};
                if (!as.intersects(lo, 8)) continue;
                if (!bit(b, lower + kLowerChildMask, m)) {
                    as.fill(lo, 8, as.tile(make_tile(rd<float>(b, lower + kLowerTable + 8 * m),
                                                     bit(b, lower + kLowerValueMask, m), 1, lower_box)));
                    continue;
                }
                const size_t leaf = lower + (size_t)rd<int64_t>(b, lower + kLowerTable + 8 * m);
                if (leaf + kLeafSize > bytes) {
                    err = "truncated NanoVDB buffer (leaf)";
                    return false;
                }
                const uint32_t idx = (uint32_t)h.leaf_src.size();
                if (idx >= kSparseTileBit) {
                    err = "too many leaves";
                    return false;
                }
                h.leaf_src.push_back(leaf);
                for (int i = 0; i < 3; i++) h.leaf_bbox_min.push_back(rd<int32_t>(b, leaf + 4 * i));
                as.fill(lo, 8, idx);
            }
        }
    }
    return true;
}

// ---------------------------------------------------------------------------------------------
// Device side

namespace {

template <class T>
cudaError_t upload(T** dst, const std::vector<T>& src, cudaStream_t s, size_t& bytes) {
    *dst = nullptr;
    if (src.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), src.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    bytes += src.size() * sizeof(T);
    return cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

cudaError_t alloc_pools(size_t leaves, bool fp16, SparseDevice& d) {
    d.leaves = leaves;
    if (leaves == 0) return cudaSuccess;
    cudaError_t e = fp16 ? cudaMalloc(reinterpret_cast<void**>(&d.values_h), leaves * 512 * sizeof(unsigned short))
                         : cudaMalloc(reinterpret_cast<void**>(&d.values), leaves * 512 * sizeof(float));
    if (e != cudaSuccess) return e;
    d.bytes += leaves * 512 * (fp16 ? 2 : 4);
    e = cudaMalloc(reinterpret_cast<void**>(&d.masks), leaves * 16 * sizeof(uint32_t));
    d.bytes += leaves * 64;
    return e;
}

// One warp per leaf: 512 values (16 per lane, coalesced) and 16 mask words.
__global__ void gather_nanovdb_leaves_kernel(const uint8_t* __restrict__ buf, const uint64_t* __restrict__ src,
                                             size_t leaves, float* __restrict__ values,
                                             unsigned short* __restrict__ values_h, uint32_t* __restrict__ masks) {
    const size_t leaf = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (leaf >= leaves) return;
    const uint8_t* node = buf + src[leaf];
    const float* v = reinterpret_cast<const float*>(node + kLeafValues);
    for (int k = lane; k < 512; k += 32) {
        const float x = v[k];
        if (values) values[leaf * 512 + k] = x;
        else values_h[leaf * 512 + k] = __half_as_ushort(__float2half_rn(x));
    }
    if (lane < 16) masks[leaf * 16 + lane] = reinterpret_cast<const uint32_t*>(node + kLeafValueMask)[lane];
}

}  // namespace

cudaError_t upload_sparse_from_nanovdb(const SparseHost& h, const uint8_t* dev_buf, bool fp16, SparseDevice& d,
                                       cudaStream_t s) {
    d.release();
    cudaError_t e = upload(&d.table, h.table, s, d.bytes);
    if (e == cudaSuccess) e = upload(&d.tiles, h.tiles, s, d.bytes);
    if (e == cudaSuccess) e = upload(&d.leaf_bbox_min, h.leaf_bbox_min, s, d.bytes);
    if (e == cudaSuccess) e = alloc_pools(h.leaf_count(), fp16, d);
    uint64_t* src = nullptr;
    if (e == cudaSuccess && d.leaves) {
        e = cudaMalloc(reinterpret_cast<void**>(&src), d.leaves * sizeof(uint64_t));
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(src, h.leaf_src.data(), d.leaves * sizeof(uint64_t), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) {
            const unsigned blocks = (unsigned)((d.leaves * 32 + 255) / 256);
            gather_nanovdb_leaves_kernel<<<blocks, 256, 0, s>>>(dev_buf, src, d.leaves, d.values, d.values_h, d.masks);
            count_launches(1);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaFree(src);
    }
    if (e != cudaSuccess) d.release();
    return e;
}

// ---------------------------------------------------------------------------------------------
// Dense -> sparse (GridBuilder semantics)

namespace {

struct BrickSummary {
    int count;        // active voxels (value != 0) inside the grid
    float v0;         // value of the brick's first voxel (LeafNode::getFirstValue)
    int all_equal;    // all 512 voxels active and equal to v0
    uint8_t mn[3], mx[3];  // per-axis min/max local coordinate of the active voxels
    uint8_t pad[2];
};

// One warp per 8^3 brick of the dense grid; lanes read two x-rows of 8 voxels each.
__global__ void brick_summary_kernel(const float* __restrict__ dense, int nx, int ny, int nz, int bx, int by,
                                     size_t bricks, BrickSummary* __restrict__ out) {
    const size_t brick = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (brick >= bricks) return;
    const int ox = (int)(brick % (size_t)bx) * 8;
    const int oy = (int)((brick / (size_t)bx) % (size_t)by) * 8;
    const int oz = (int)(brick / ((size_t)bx * by)) * 8;
    const float v0 = dense[((size_t)oz * ny + oy) * nx + ox];
    int count = 0;
    bool eq = true;
    unsigned mn[3] = {8u, 8u, 8u}, mx[3] = {0u, 0u, 0u};
    for (int r = lane; r < 64; r += 32) {
        const int ly = r & 7, lz = r >> 3;
        const int y = oy + ly, z = oz + lz;
        for (int lx = 0; lx < 8; lx++) {
            const int x = ox + lx;
            const bool in = x < nx && y < ny && z < nz;
            const float v = in ? dense[((size_t)z * ny + y) * nx + x] : 0.0f;
            const bool act = in && v != 0.0f;
            if (act) {
                count++;
                mn[0] = min(mn[0], (unsigned)lx); mx[0] = max(mx[0], (unsigned)lx);
                mn[1] = min(mn[1], (unsigned)ly); mx[1] = max(mx[1], (unsigned)ly);
                mn[2] = min(mn[2], (unsigned)lz); mx[2] = max(mx[2], (unsigned)lz);
            }
            eq = eq && act && v == v0;
        }
    }
    count = (int)__reduce_add_sync(0xffffffffu, (unsigned)count);
    const bool all_eq = __all_sync(0xffffffffu, eq);
    for (int a = 0; a < 3; a++) {
        mn[a] = __reduce_min_sync(0xffffffffu, mn[a]);
        mx[a] = __reduce_max_sync(0xffffffffu, mx[a]);
    }
    if (lane == 0) {
        BrickSummary s;
        s.count = count;
        s.v0 = v0;
        s.all_equal = (all_eq && count == 512) ? 1 : 0;
        for (int a = 0; a < 3; a++) {
            s.mn[a] = (uint8_t)mn[a];
            s.mx[a] = (uint8_t)mx[a];
        }
        s.pad[0] = s.pad[1] = 0;
        out[brick] = s;
    }
}

// One warp per leaf: values in NanoVDB voxel order and the active mask, from the dense grid.
__global__ void gather_dense_leaves_kernel(const float* __restrict__ dense, int nx, int ny, int nz, int bx, int by,
                                           const uint64_t* __restrict__ src, size_t leaves, float* __restrict__ values,
                                           unsigned short* __restrict__ values_h, uint32_t* __restrict__ masks) {
    const size_t leaf = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (leaf >= leaves) return;
    const size_t brick = src[leaf];
    const int ox = (int)(brick % (size_t)bx) * 8;
    const int oy = (int)((brick / (size_t)bx) % (size_t)by) * 8;
    const int oz = (int)(brick / ((size_t)bx * by)) * 8;
    for (int k = lane; k < 512; k += 32) {
        const int x = ox + (k >> 6), y = oy + ((k >> 3) & 7), z = oz + (k & 7);
        const bool in = x < nx && y < ny && z < nz;
        const float v = in ? dense[((size_t)z * ny + y) * nx + x] : 0.0f;
        if (values) values[leaf * 512 + k] = v;
        else values_h[leaf * 512 + k] = __half_as_ushort(__float2half_rn(v));
        const unsigned ballot = __ballot_sync(0xffffffffu, in && v != 0.0f);
        if (lane == 0) masks[leaf * 16 + (k >> 5)] = ballot;
    }
}

struct Box {
    int lo[3] = {INT_MAX, INT_MAX, INT_MAX};
    int hi[3] = {INT_MIN, INT_MIN, INT_MIN};
    void add(const int* a, const int* b) {
        for (int i = 0; i < 3; i++) {
            lo[i] = std::min(lo[i], a[i]);
            hi[i] = std::max(hi[i], b[i]);
        }
    }
    void add(const Box& o) {
        if (!o.empty()) add(o.lo, o.hi);
    }
    bool empty() const { return lo[0] > hi[0] || lo[1] > hi[1] || lo[2] > hi[2]; }
    void out(int* box) const {
        for (int i = 0; i < 3; i++) {
            box[i] = lo[i];
            box[3 + i] = hi[i];
        }
    }
};

}  // namespace

cudaError_t build_sparse_from_dense(const float* dense, int nx, int ny, int nz, double dx, const double origin[3],
                                    bool fp16, SparseHost& h, SparseDevice& d, cudaStream_t s, std::string& err) {
    h = SparseHost();
    d.release();
    const int bx = (nx + 7) / 8, by = (ny + 7) / 8, bz = (nz + 7) / 8;
    const size_t bricks = (size_t)bx * by * bz;
    std::vector<BrickSummary> sum(bricks);
    {
        BrickSummary* dsum = nullptr;
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&dsum), bricks * sizeof(BrickSummary));
        if (e != cudaSuccess) return e;
        brick_summary_kernel<<<(unsigned)((bricks * 32 + 255) / 256), 256, 0, s>>>(dense, nx, ny, nz, bx, by, bricks,
                                                                                  dsum);
        count_launches(1);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sum.data(), dsum, bricks * sizeof(BrickSummary), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaFree(dsum);
        if (e != cudaSuccess) return e;
    }
    // Map (GridBuilder::getHandle(dx, origin), GridBuilder.h:535-559; Map::set, NanoVDB.h:2043-2060).
    for (int i = 0; i < 9; i++) {
        h.mat[i] = (i % 4 == 0) ? (float)dx : 0.0f;
        h.inv_mat[i] = (i % 4 == 0) ? (float)(1.0 / dx) : 0.0f;
    }
    for (int i = 0; i < 3; i++) {
        h.vec[i] = (float)origin[i];
        h.voxel_size[i] = dx;
    }
    h.background = 0.0f;

    // Node hierarchy.  Lower nodes are 16^3 bricks, upper nodes 32^3 lower nodes.
    const int lx = (bx + 15) / 16, ly = (by + 15) / 16, lz = (bz + 15) / 16;
    const int ux = (lx + 31) / 32, uy = (ly + 31) / 32, uz = (lz + 31) / 32;
    auto bidx = [&](int x, int y, int z) { return ((size_t)z * by + y) * bx + x; };
    auto status = [&](int x, int y, int z) -> int {  // 0 empty, 1 leaf, 2 pruned to an active tile
        if (x >= bx || y >= by || z >= bz) return 0;
        const BrickSummary& b = sum[bidx(x, y, z)];
        if (b.count == 0) return 0;
        return b.all_equal ? 2 : 1;
    };
    const size_t nlower = (size_t)lx * ly * lz;
    std::vector<uint8_t> lower_exists(nlower, 0), lower_pruned(nlower, 0);
    std::vector<float> lower_value(nlower, 0.0f);
    std::vector<Box> lower_box(nlower);
    for (int z = 0; z < lz; z++)
        for (int y = 0; y < ly; y++)
            for (int x = 0; x < lx; x++) {
                const size_t li = ((size_t)z * ly + y) * lx + x;
                bool any = false, all_tiles = true, same = true;
                float first = 0.0f;
                bool have_first = false;
                Box box;
                for (int k = 0; k < 16; k++)
                    for (int j = 0; j < 16; j++)
                        for (int i = 0; i < 16; i++) {
                            const int gx = x * 16 + i, gy = y * 16 + j, gz = z * 16 + k;
                            const int st = status(gx, gy, gz);
                            const float v = st == 2 ? sum[bidx(gx, gy, gz)].v0 : 0.0f;
                            if (!have_first) {
                                first = v;
                                have_first = true;
                            } else if (v != first) {
                                same = false;
                            }
                            if (st == 0) continue;
                            any = true;
                            const BrickSummary& b = sum[bidx(gx, gy, gz)];
                            const int o[3] = {gx * 8, gy * 8, gz * 8};
                            if (st == 1) {
                                all_tiles = false;
                                const int a[3] = {o[0] + b.mn[0], o[1] + b.mn[1], o[2] + b.mn[2]};
                                const int c[3] = {o[0] + b.mx[0], o[1] + b.mx[1], o[2] + b.mx[2]};
                                box.add(a, c);
                            } else {
                                const int c[3] = {o[0] + 7, o[1] + 7, o[2] + 7};
                                box.add(o, c);
                            }
                        }
                lower_exists[li] = any;
                lower_pruned[li] = any && all_tiles && same;
                lower_value[li] = first;
                lower_box[li] = box;
            }
    const size_t nupper = (size_t)ux * uy * uz;
    std::vector<uint8_t> upper_exists(nupper, 0), upper_pruned(nupper, 0);
    std::vector<float> upper_value(nupper, 0.0f);
    std::vector<Box> upper_box(nupper);
    Box root_box;
    for (int z = 0; z < uz; z++)
        for (int y = 0; y < uy; y++)
            for (int x = 0; x < ux; x++) {
                const size_t ui = ((size_t)z * uy + y) * ux + x;
                bool any = false, all_pruned = true, same = true, have_first = false;
                float first = 0.0f;
                Box box;
                for (int k = 0; k < 32; k++)
                    for (int j = 0; j < 32; j++)
                        for (int i = 0; i < 32; i++) {
                            const int gx = x * 32 + i, gy = y * 32 + j, gz = z * 32 + k;
                            bool ex = false, pr = false;
                            float v = 0.0f;
                            size_t li = 0;
                            if (gx < lx && gy < ly && gz < lz) {
                                li = ((size_t)gz * ly + gy) * lx + gx;
                                ex = lower_exists[li];
                                pr = lower_pruned[li];
                                v = pr ? lower_value[li] : 0.0f;
                            }
                            if (!have_first) {
                                first = v;
                                have_first = true;
                            } else if (v != first) {
                                same = false;
                            }
                            if (!ex) continue;
                            any = true;
                            if (pr) {
                                const int o[3] = {gx * 128, gy * 128, gz * 128};
                                const int c[3] = {o[0] + 127, o[1] + 127, o[2] + 127};
                                box.add(o, c);
                            } else {
                                all_pruned = false;
                                box.add(lower_box[li]);
                            }
                        }
                upper_exists[ui] = any;
                upper_pruned[ui] = any && all_pruned && same;
                upper_value[ui] = first;
                if (upper_pruned[ui]) {
                    const int o[3] = {x * 4096, y * 4096, z * 4096};
                    const int c[3] = {o[0] + 4095, o[1] + 4095, o[2] + 4095};
                    Box rb;
                    rb.add(o, c);
                    root_box.add(rb);
                } else {
                    root_box.add(box);
                }
                upper_box[ui] = box;
            }
    if (!root_box.empty()) {
        for (int i = 0; i < 3; i++) {
            h.root_min[i] = root_box.lo[i];
            h.root_max[i] = root_box.hi[i];
        }
        // World box: Map::applyMap in double on the index box corners, max + 1 (GridStats.h:536-560).
        for (int i = 0; i < 3; i++) {
            h.world_min[i] = fma((double)h.root_min[i], dx, origin[i]);
            h.world_max[i] = fma((double)h.root_max[i] + 1.0, dx, origin[i]);
        }
    }
    Assembler as(h);
    if (!as.init_table(err)) return cudaErrorInvalidValue;
    int root_b[6];
    root_box.out(root_b);
    for (int z = 0; z < uz; z++)
        for (int y = 0; y < uy; y++)
            for (int x = 0; x < ux; x++) {
                const size_t ui = ((size_t)z * uy + y) * ux + x;
                if (!upper_exists[ui]) continue;
                const long long uo[3] = {x * 4096LL, y * 4096LL, z * 4096LL};
                h.root_tiles.push_back({{(int)uo[0], (int)uo[1], (int)uo[2]}, upper_pruned[ui] ? 0 : 1,
                                        upper_pruned[ui] ? upper_value[ui] : 0.0f, upper_pruned[ui] ? 1 : 0});
                if (upper_pruned[ui]) {
                    as.fill(uo, 4096, as.tile(make_tile(upper_value[ui], true, 3, root_b)));
                    continue;
                }
                int ub[6];
                upper_box[ui].out(ub);
                for (int k = 0; k < 32; k++)
                    for (int j = 0; j < 32; j++)
                        for (int i = 0; i < 32; i++) {
                            const long long lo[3] = {uo[0] + i * 128LL, uo[1] + j * 128LL, uo[2] + k * 128LL};
                            if (!as.intersects(lo, 128)) continue;
                            const int gx = x * 32 + i, gy = y * 32 + j, gz = z * 32 + k;
                            const bool in = gx < lx && gy < ly && gz < lz;
                            const size_t li = in ? ((size_t)gz * ly + gy) * lx + gx : 0;
                            if (!in || !lower_exists[li]) {
                                as.fill(lo, 128, as.tile(make_tile(0.0f, false, 2, ub)));
                                continue;
                            }
                            if (lower_pruned[li]) {
                                as.fill(lo, 128, as.tile(make_tile(lower_value[li], true, 2, ub)));
                                continue;
                            }
                            int lb[6];
                            lower_box[li].out(lb);
                            for (int c = 0; c < 16; c++)
                                for (int bb = 0; bb < 16; bb++)
                                    for (int a = 0; a < 16; a++) {
                                        const int gbx = gx * 16 + a, gby = gy * 16 + bb, gbz = gz * 16 + c;
                                        const long long o[3] = {gbx * 8LL, gby * 8LL, gbz * 8LL};
                                        const int st = status(gbx, gby, gbz);
                                        if (st == 1) {
                                            const BrickSummary& b = sum[bidx(gbx, gby, gbz)];
                                            const uint32_t idx = (uint32_t)h.leaf_src.size();
                                            h.leaf_src.push_back(bidx(gbx, gby, gbz));
                                            h.leaf_bbox_min.push_back((int)o[0] + b.mn[0]);
                                            h.leaf_bbox_min.push_back((int)o[1] + b.mn[1]);
                                            h.leaf_bbox_min.push_back((int)o[2] + b.mn[2]);
                                            as.fill(o, 8, idx);
                                        } else if (st == 2) {
                                            as.fill(o, 8, as.tile(make_tile(sum[bidx(gbx, gby, gbz)].v0, true, 1, lb)));
                                        } else {
                                            as.fill(o, 8, as.tile(make_tile(0.0f, false, 1, lb)));
                                        }
                                    }
                        }
            }
    cudaError_t e = upload(&d.table, h.table, s, d.bytes);
    if (e == cudaSuccess) e = upload(&d.tiles, h.tiles, s, d.bytes);
    if (e == cudaSuccess) e = upload(&d.leaf_bbox_min, h.leaf_bbox_min, s, d.bytes);
    if (e == cudaSuccess) e = alloc_pools(h.leaf_count(), fp16, d);
    if (e == cudaSuccess && d.leaves) {
        uint64_t* src = nullptr;
        e = cudaMalloc(reinterpret_cast<void**>(&src), d.leaves * sizeof(uint64_t));
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(src, h.leaf_src.data(), d.leaves * sizeof(uint64_t), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) {
            gather_dense_leaves_kernel<<<(unsigned)((d.leaves * 32 + 255) / 256), 256, 0, s>>>(
                dense, nx, ny, nz, bx, by, src, d.leaves, d.values, d.values_h, d.masks);
            count_launches(1);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaFree(src);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) d.release();
    return e;
}

SparseView make_sparse_view(const SparseHost& h, const SparseDevice& d, int lowest_level) {
    SparseView v{};
    memcpy(v.mat, h.mat, sizeof(v.mat));
    memcpy(v.inv_mat, h.inv_mat, sizeof(v.inv_mat));
    memcpy(v.vec, h.vec, sizeof(v.vec));
    v.grid_min = F3{(float)h.world_min[0], (float)h.world_min[1], (float)h.world_min[2]};
    v.grid_max = F3{(float)h.world_max[0], (float)h.world_max[1], (float)h.world_max[2]};
    for (int i = 0; i < 3; i++) {
        v.root_min[i] = h.root_min[i];
        v.root_max[i] = h.root_max[i];
        v.tbl_origin[i] = h.tbl_origin[i];
        v.tbl_dim[i] = h.tbl_dim[i];
    }
    v.lowest_level = lowest_level;
    v.fp16 = d.values_h != nullptr;
    v.background = h.background;
    v.root_tiles = (int)std::min<size_t>(h.root_tiles.size(), kSparseMaxRootTiles);
    for (int t = 0; t < v.root_tiles; t++) {
        for (int i = 0; i < 3; i++) v.rt_origin[t][i] = h.root_tiles[t].origin[i];
        v.rt_child[t] = h.root_tiles[t].child;
        v.rt_value[t] = h.root_tiles[t].value;
        v.rt_active[t] = h.root_tiles[t].active;
    }
    v.table = d.table;
    v.values = d.values;
    v.values_h = d.values_h;
    v.masks = d.masks;
    v.leaf_bbox_min = d.leaf_bbox_min;
    v.tiles = d.tiles;
    return v;
}

}  // namespace vpt
