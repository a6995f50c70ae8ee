// vpt_sparse.cuh - device side of sparse (NanoVDB-compatible) volumes: map, brick-table lookups,
// the three interpolations of sampleCloudRaw for NanoVDB (VptUtils.glsl:496-581), the hierarchical
// DDA of PNanoVDB.glsl:2233-2452 and the sparse decomposition tracker
// (DecompositionTracking.glsl:130-360).
//
// The tree is read through the flattened brick table of SparseView (vpt_params.h): one 32-bit load
// per lookup finds the leaf (then one load of the voxel) or the constant tile of the brick.  The
// values, activity, node levels and node boxes it returns are those of the NanoVDB tree it was
// built from; the CPU oracle checks them against the reference's PNanoVDB accessor.
#pragma once
#include <cuda_fp16.h>
#include "vpt_device.cuh"

namespace vpt {

// pnanovdb_map_apply_inverse / _inverse_jacobi / _apply (PNanoVDB.glsl:1996-2040): float, rows in
// the order PNanoVDB sums them.
VPT_DEV F3 sparse_world_to_index(const SparseView& S, F3 p) {
    const float sx = p.x - S.vec[0], sy = p.y - S.vec[1], sz = p.z - S.vec[2];
    return f3((sx * S.inv_mat[0] + sy * S.inv_mat[1]) + sz * S.inv_mat[2],
              (sx * S.inv_mat[3] + sy * S.inv_mat[4]) + sz * S.inv_mat[5],
              (sx * S.inv_mat[6] + sy * S.inv_mat[7]) + sz * S.inv_mat[8]);
}
VPT_DEV F3 sparse_world_to_index_dir(const SparseView& S, F3 d) {
    return f3((d.x * S.inv_mat[0] + d.y * S.inv_mat[1]) + d.z * S.inv_mat[2],
              (d.x * S.inv_mat[3] + d.y * S.inv_mat[4]) + d.z * S.inv_mat[5],
              (d.x * S.inv_mat[6] + d.y * S.inv_mat[7]) + d.z * S.inv_mat[8]);
}
VPT_DEV F3 sparse_index_to_world(const SparseView& S, F3 p) {
    return f3(((p.x * S.mat[0] + p.y * S.mat[1]) + p.z * S.mat[2]) + S.vec[0],
              ((p.x * S.mat[3] + p.y * S.mat[4]) + p.z * S.mat[5]) + S.vec[1],
              ((p.x * S.mat[6] + p.y * S.mat[7]) + p.z * S.mat[8]) + S.vec[2]);
}

// Table entry of the brick holding voxel (x, y, z); false outside the table (background).
VPT_DEV bool sparse_entry(const SparseView& S, int x, int y, int z, uint32_t& e) {
    const int bx = (x - S.tbl_origin[0]) >> 3;
    const int by = (y - S.tbl_origin[1]) >> 3;
    const int bz = (z - S.tbl_origin[2]) >> 3;
    if ((unsigned)bx >= (unsigned)S.tbl_dim[0] || (unsigned)by >= (unsigned)S.tbl_dim[1] ||
        (unsigned)bz >= (unsigned)S.tbl_dim[2])
        return false;
    e = __ldg(S.table + ((size_t)bz * (unsigned)S.tbl_dim[1] + (unsigned)by) * (unsigned)S.tbl_dim[0] + (unsigned)bx);
    return true;
}

// Root tile holding a voxel outside the brick table (-1: none).
VPT_DEV int sparse_root_tile(const SparseView& S, int x, int y, int z) {
    const int ox = x & ~4095, oy = y & ~4095, oz = z & ~4095;
    for (int t = 0; t < S.root_tiles; t++)
        if (S.rt_origin[t][0] == ox && S.rt_origin[t][1] == oy && S.rt_origin[t][2] == oz) return t;
    return -1;
}

VPT_DEV uint32_t sparse_leaf_offset(int x, int y, int z) {
    return ((uint32_t)(x & 7) << 6) | ((uint32_t)(y & 7) << 3) | (uint32_t)(z & 7);
}

// pnanovdb_readaccessor_get_value_address + pnanovdb_read_float.
VPT_DEV float sparse_value(const SparseView& S, int x, int y, int z) {
    uint32_t e;
    if (!sparse_entry(S, x, y, z, e)) {
        const int t = sparse_root_tile(S, x, y, z);
        return (t >= 0 && !S.rt_child[t]) ? S.rt_value[t] : S.background;
    }
    if (e & kSparseTileBit) return S.tiles[e & ~kSparseTileBit].value;
    const size_t i = (size_t)e * 512u + sparse_leaf_offset(x, y, z);
    return S.fp16 ? __half2float(__ushort_as_half(__ldg(S.values_h + i))) : __ldg(S.values + i);
}

// pnanovdb_readaccessor_get_dim: 1 inside a leaf, 8 / 128 / 4096 for lower / upper / root tiles and
// the background.
VPT_DEV int sparse_dim(const SparseView& S, int x, int y, int z) {
    uint32_t e;
    if (!sparse_entry(S, x, y, z, e)) {
        const int t = sparse_root_tile(S, x, y, z);
        return (t >= 0 && S.rt_child[t]) ? 128 : 4096;
    }
    if (!(e & kSparseTileBit)) return 1;
    const int level = S.tiles[e & ~kSparseTileBit].level;
    return level == 1 ? 8 : (level == 2 ? 128 : 4096);
}

// pnanovdb_readaccessor_is_active.
VPT_DEV bool sparse_is_active(const SparseView& S, int x, int y, int z) {
    uint32_t e;
    if (!sparse_entry(S, x, y, z, e)) {
        const int t = sparse_root_tile(S, x, y, z);
        return t >= 0 && !S.rt_child[t] && S.rt_active[t];
    }
    if (e & kSparseTileBit) return S.tiles[e & ~kSparseTileBit].active != 0;
    const uint32_t n = sparse_leaf_offset(x, y, z);
    return (__ldg(S.masks + (size_t)e * 16u + (n >> 5)) >> (n & 31u)) & 1u;
}

VPT_DEV int floor_to_int(float v) { return (int)floorf(v); }

// sampleCloud (VptUtils.glsl:674-683: render box -> grid world box) + sampleCloudRaw for NanoVDB
// (VptUtils.glsl:517-581).
template <int INTERP>
VPT_DEV float sample_sparse(const TraceParams& P, F3 pos, Rng& rng) {
    const SparseView& S = P.sparse;
    F3 c;
    c.x = ((pos.x - P.box_min.x) / (P.box_max.x - P.box_min.x)) * (S.grid_max.x - S.grid_min.x) + S.grid_min.x;
    c.y = ((pos.y - P.box_min.y) / (P.box_max.y - P.box_min.y)) * (S.grid_max.y - S.grid_min.y) + S.grid_min.y;
    c.z = ((pos.z - P.box_min.z) / (P.box_max.z - P.box_min.z)) * (S.grid_max.z - S.grid_min.z) + S.grid_min.z;
    F3 p = sparse_world_to_index(S, c);
    if (INTERP == kNearest) {
        return sparse_value(S, floor_to_int(p.x), floor_to_int(p.y), floor_to_int(p.z));
    } else if (INTERP == kStochastic) {
        const float jx = rng_next(rng) - 0.5f;
        const float jy = rng_next(rng) - 0.5f;
        const float jz = rng_next(rng) - 0.5f;
        return sparse_value(S, floor_to_int(p.x + jx), floor_to_int(p.y + jy), floor_to_int(p.z + jz));
    } else {
        p = f3(p.x - 0.5f, p.y - 0.5f, p.z - 0.5f);
        const int ix = floor_to_int(p.x), iy = floor_to_int(p.y), iz = floor_to_int(p.z);
        const float fx = p.x - (float)ix, fy = p.y - (float)iy, fz = p.z - (float)iz;
        const float f00 = mixf(sparse_value(S, ix, iy, iz), sparse_value(S, ix + 1, iy, iz), fx);
        const float f10 = mixf(sparse_value(S, ix, iy + 1, iz), sparse_value(S, ix + 1, iy + 1, iz), fx);
        const float f0 = mixf(f00, f10, fy);
        const float f01 = mixf(sparse_value(S, ix, iy, iz + 1), sparse_value(S, ix + 1, iy, iz + 1), fx);
        const float f11 = mixf(sparse_value(S, ix, iy + 1, iz + 1), sparse_value(S, ix + 1, iy + 1, iz + 1), fx);
        const float f1 = mixf(f01, f11, fy);
        return mixf(f0, f1, fz);
    }
}

// ---------------------------------------------------------------------------------------------
// Hierarchical DDA (pnanovdb_hdda_*, PNanoVDB.glsl:2233-2452).

struct Hdda {
    int dim;
    float tmin, tmax;
    int voxel[3];
    int step[3];
    float delta[3];
    float next[3];
};

VPT_DEV float pn_min(float a, float b) { return a < b ? a : b; }
VPT_DEV float pn_max(float a, float b) { return a > b ? a : b; }

VPT_DEV bool hdda_ray_clip(F3 bmin, F3 bmax, F3 origin, float& tmin, F3 direction, float& tmax) {
    const F3 inv = f3(1.0f / direction.x, 1.0f / direction.y, 1.0f / direction.z);
    const F3 t0 = f3((bmin.x - origin.x) * inv.x, (bmin.y - origin.y) * inv.y, (bmin.z - origin.z) * inv.z);
    const F3 t1 = f3((bmax.x - origin.x) * inv.x, (bmax.y - origin.y) * inv.y, (bmax.z - origin.z) * inv.z);
    const float tnear = pn_max(pn_min(t0.x, t1.x), pn_max(pn_min(t0.y, t1.y), pn_min(t0.z, t1.z)));
    const float tfar = pn_min(pn_max(t0.x, t1.x), pn_min(pn_max(t0.y, t1.y), pn_max(t0.z, t1.z)));
    const bool hit = tnear <= tfar;
    tmin = pn_max(tmin, tnear);
    tmax = pn_min(tmax, tfar);
    return hit;
}

VPT_DEV void hdda_axis_init(Hdda& h, int a, float o, float d, float pos, float inv) {
    if (d == 0.0f) {
        h.next[a] = 1e38f;
        h.step[a] = 0;
        h.delta[a] = 0.0f;
    } else if (inv > 0.0f) {
        h.step[a] = 1;
        h.next[a] = h.tmin + ((float)(h.voxel[a] + h.dim) - pos) * inv;
        h.delta[a] = inv;
    } else {
        h.step[a] = -1;
        h.next[a] = h.tmin + ((float)h.voxel[a] - pos) * inv;
        h.delta[a] = -inv;
    }
}

VPT_DEV void hdda_init(Hdda& h, F3 origin, float tmin, F3 direction, float tmax, int dim) {
    h.dim = dim;
    h.tmin = tmin;
    h.tmax = tmax;
    const F3 pos = f3(direction.x * tmin + origin.x, direction.y * tmin + origin.y, direction.z * tmin + origin.z);
    const F3 inv = f3(1.0f / direction.x, 1.0f / direction.y, 1.0f / direction.z);
    h.voxel[0] = floor_to_int(pos.x) & ~(dim - 1);
    h.voxel[1] = floor_to_int(pos.y) & ~(dim - 1);
    h.voxel[2] = floor_to_int(pos.z) & ~(dim - 1);
    hdda_axis_init(h, 0, origin.x, direction.x, pos.x, inv.x);
    hdda_axis_init(h, 1, origin.y, direction.y, pos.y, inv.y);
    hdda_axis_init(h, 2, origin.z, direction.z, pos.z, inv.z);
}

VPT_DEV bool hdda_update(Hdda& h, F3 origin, F3 direction, int dim) {
    if (h.dim == dim) return false;
    h.dim = dim;
    const F3 pos = f3(direction.x * h.tmin + origin.x, direction.y * h.tmin + origin.y, direction.z * h.tmin + origin.z);
    const float inv[3] = {1.0f / direction.x, 1.0f / direction.y, 1.0f / direction.z};
    const float p[3] = {pos.x, pos.y, pos.z};
    for (int a = 0; a < 3; a++) h.voxel[a] = floor_to_int(p[a]) & ~(dim - 1);
    for (int a = 0; a < 3; a++) {
        if (h.step[a] != 0) {
            h.next[a] = h.tmin + ((float)h.voxel[a] - p[a]) * inv[a];
            if (h.step[a] > 0) h.next[a] += (float)dim * inv[a];
        }
    }
    return true;
}

VPT_DEV bool hdda_step(Hdda& h) {
    int a;
    if (h.next[0] < h.next[1] && h.next[0] < h.next[2]) a = 0;
    else if (h.next[1] < h.next[2]) a = 1;
    else a = 2;
    if (h.next[a] <= h.tmin) h.next[a] += (h.tmin - 0.999999f * h.next[a]) + 1.0e-6f;
    h.tmin = h.next[a];
    h.next[a] += (float)h.dim * h.delta[a];
    h.voxel[a] += h.dim * h.step[a];
    return h.tmin <= h.tmax;
}

// Node of the HDDA cell at `v` as the sparse decomposition tracker classifies it
// (DecompositionTracking.glsl:178-248): active flag and node box in index space.
VPT_DEV bool sparse_cell_node(const SparseView& S, const int v[3], F3& bmin, F3& bmax) {
    if (S.lowest_level != 8) {
        bmin = f3((float)v[0], (float)v[1], (float)v[2]);
        bmax = f3((float)(v[0] + 1), (float)(v[1] + 1), (float)(v[2] + 1));
        return sparse_is_active(S, v[0], v[1], v[2]);
    }
    uint32_t e;
    if (!sparse_entry(S, v[0], v[1], v[2], e)) {
        const int t = sparse_root_tile(S, v[0], v[1], v[2]);
        if (t < 0 || S.rt_child[t] || !S.rt_active[t]) return false;
        bmin = f3((float)S.root_min[0], (float)S.root_min[1], (float)S.root_min[2]);
        bmax = f3((float)S.root_max[0], (float)S.root_max[1], (float)S.root_max[2]);
        return true;
    }
    if (!(e & kSparseTileBit)) {
        const int* b = S.leaf_bbox_min + (size_t)e * 3u;
        bmin = f3((float)b[0], (float)b[1], (float)b[2]);
        bmax = f3((float)(b[0] + 8), (float)(b[1] + 8), (float)(b[2] + 8));
        return true;
    }
    const SparseTile& t = S.tiles[e & ~kSparseTileBit];
    if (t.level > 3 || !t.active) return false;
    bmin = f3((float)t.box[0], (float)t.box[1], (float)t.box[2]);
    bmax = f3((float)t.box[3], (float)t.box[4], (float)t.box[5]);
    return true;
}

}  // namespace vpt
