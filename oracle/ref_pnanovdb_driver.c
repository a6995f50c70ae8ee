/* ref_pnanovdb_driver.c - TEST INFRASTRUCTURE ONLY.  Compiled by oracle/ref_build.py together with
 * the reference's Data/Shaders/VPT/PNanoVDB.glsl in its own C mode (-DPNANOVDB_C -DPNANOVDB_HDDA);
 * the output library lives in oracle/_ref/.  It exposes the reference's NanoVDB read accessor, map
 * and HDDA on a grid buffer, so that the oracle's restatement and the CUDA core's sparse volume can
 * be checked against them bit for bit. */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define PNANOVDB_C
#define PNANOVDB_HDDA
#include "PNanoVDB.glsl"

static pnanovdb_buf_t make_buf(const uint32_t* data) {
    pnanovdb_buf_t b;
    b.data = (uint32_t*)data;
    return b;
}

static pnanovdb_root_handle_t root_of(pnanovdb_buf_t buf) {
    pnanovdb_grid_handle_t grid;
    grid.address = pnanovdb_address_null();
    return pnanovdb_tree_get_root(buf, pnanovdb_grid_get_tree(buf, grid));
}

/* Value, get_dim and is_active of a list of voxels, through one read accessor that keeps its
 * cache from query to query (as a shader invocation does). */
void refvdb_query(const uint32_t* data, int n, const int32_t* ijk, float* value, uint32_t* dim, uint8_t* active) {
    pnanovdb_buf_t buf = make_buf(data);
    pnanovdb_readaccessor_t acc;
    pnanovdb_readaccessor_init(&acc, root_of(buf));
    for (int i = 0; i < n; i++) {
        pnanovdb_coord_t c;
        c.x = ijk[3 * i];
        c.y = ijk[3 * i + 1];
        c.z = ijk[3 * i + 2];
        pnanovdb_address_t a = pnanovdb_readaccessor_get_value_address(PNANOVDB_GRID_TYPE_FLOAT, buf, &acc, &c);
        value[i] = pnanovdb_read_float(buf, a);
        dim[i] = pnanovdb_readaccessor_get_dim(PNANOVDB_GRID_TYPE_FLOAT, buf, &acc, &c);
        active[i] = (uint8_t)pnanovdb_readaccessor_is_active(PNANOVDB_GRID_TYPE_FLOAT, buf, &acc, &c);
    }
}

/* pnanovdb_grid_world_to_indexf / _dirf / index_to_worldf on a list of points. */
void refvdb_map(const uint32_t* data, int n, int which, const float* in, float* out) {
    pnanovdb_buf_t buf = make_buf(data);
    pnanovdb_grid_handle_t grid;
    grid.address = pnanovdb_address_null();
    for (int i = 0; i < n; i++) {
        pnanovdb_vec3_t v;
        v.x = in[3 * i];
        v.y = in[3 * i + 1];
        v.z = in[3 * i + 2];
        pnanovdb_vec3_t r;
        if (which == 0) r = pnanovdb_grid_world_to_indexf(buf, grid, &v);
        else if (which == 1) r = pnanovdb_grid_world_to_index_dirf(buf, grid, &v);
        else r = pnanovdb_grid_index_to_worldf(buf, grid, &v);
        out[3 * i] = r.x;
        out[3 * i + 1] = r.y;
        out[3 * i + 2] = r.z;
    }
}

void refvdb_root_bbox(const uint32_t* data, int32_t out[6]) {
    pnanovdb_buf_t buf = make_buf(data);
    pnanovdb_root_handle_t root = root_of(buf);
    pnanovdb_coord_t a = pnanovdb_root_get_bbox_min(buf, root);
    pnanovdb_coord_t b = pnanovdb_root_get_bbox_max(buf, root);
    out[0] = a.x; out[1] = a.y; out[2] = a.z;
    out[3] = b.x; out[4] = b.y; out[5] = b.z;
}

/* The node walk of the sparse decomposition tracker (DecompositionTracking.glsl:130-250) for a
 * straight ray (no collision): ray set-up, root-box clip, HDDA at the lowest level, and for every
 * visited cell the node that holds it.  Per visit it records: hdda.voxel (3), dim, is_active,
 * node level (0 leaf, 1 lower, 2 upper, 3 root tile; -1 voxel level), the node box (6 floats),
 * hdda.tmin, min(hdda.next) and the clipped tMinNode.  Returns the number of visits (<= max_visits),
 * or -1 if the ray misses the root box. */
int refvdb_hdda_walk(const uint32_t* data, const float world_origin[3], const float world_dir[3], int lowest_level,
                     int max_visits, int32_t* out_voxel, int32_t* out_dim, uint8_t* out_active, int32_t* out_level,
                     float* out_box, float* out_t) {
    pnanovdb_buf_t buf = make_buf(data);
    pnanovdb_grid_handle_t grid;
    grid.address = pnanovdb_address_null();
    pnanovdb_readaccessor_t accessor;
    pnanovdb_readaccessor_init(&accessor, root_of(buf));
    pnanovdb_vec3_t x = {world_origin[0], world_origin[1], world_origin[2]};
    pnanovdb_vec3_t w = {world_dir[0], world_dir[1], world_dir[2]};
    pnanovdb_vec3_t origin = pnanovdb_grid_world_to_indexf(buf, grid, &x);
    pnanovdb_vec3_t direction = pnanovdb_grid_world_to_index_dirf(buf, grid, &w);
    float len = sqrtf(direction.x * direction.x + direction.y * direction.y + direction.z * direction.z);
    float gridToWorldScale = 1.0f / len;
    direction.x *= gridToWorldScale;
    direction.y *= gridToWorldScale;
    direction.z *= gridToWorldScale;
    float tMin = 0.0f, tMax = 1e10f;
    pnanovdb_coord_t bbox_min = pnanovdb_root_get_bbox_min(buf, accessor.root);
    pnanovdb_coord_t bbox_max = pnanovdb_root_get_bbox_max(buf, accessor.root);
    pnanovdb_vec3_t bbox_minf = pnanovdb_coord_to_vec3(bbox_min);
    pnanovdb_coord_t one = pnanovdb_coord_uniform(1);
    pnanovdb_coord_t bmax1 = pnanovdb_coord_add(bbox_max, one);
    pnanovdb_vec3_t bbox_maxf = pnanovdb_coord_to_vec3(bmax1);
    int hit = pnanovdb_hdda_ray_clip(&bbox_minf, &bbox_maxf, &origin, &tMin, &direction, &tMax);
    if (!(hit && tMax < 1e20f)) return -1;
    int dim = lowest_level;
    pnanovdb_hdda_t hdda;
    pnanovdb_hdda_init(&hdda, &origin, tMin - 1e-4f, &direction, tMax + 1e-4f, dim);
    int visits = 0;
    for (int iteration = 0; visits < max_visits; iteration++) {
        if (iteration > 0) {
            if (!pnanovdb_hdda_step(&hdda)) break;
            int d = (int)pnanovdb_readaccessor_get_dim(PNANOVDB_GRID_TYPE_FLOAT, buf, &accessor, &hdda.voxel);
            d = d > lowest_level ? d : lowest_level;
            pnanovdb_hdda_update(&hdda, &origin, &direction, d);
        }
        int level = -1;
        int isActive = 0;
        pnanovdb_vec3_t nmin, nmax;
        if (lowest_level == 8) {
            pnanovdb_root_tile_handle_t tile =
                pnanovdb_root_find_tile(PNANOVDB_GRID_TYPE_FLOAT, buf, accessor.root, &hdda.voxel);
            if (pnanovdb_address_is_null(tile.address)) {
                /* the shader reads a child offset at address 8 of the buffer here; not modelled */
                level = 4;
                isActive = 0;
            } else if (!pnanovdb_int64_is_zero(pnanovdb_root_tile_get_child(buf, tile))) {
                pnanovdb_upper_handle_t upper =
                    pnanovdb_root_get_child(PNANOVDB_GRID_TYPE_FLOAT, buf, accessor.root, tile);
                pnanovdb_uint32_t un = pnanovdb_upper_coord_to_offset(&hdda.voxel);
                if (pnanovdb_upper_get_child_mask(buf, upper, un)) {
                    pnanovdb_lower_handle_t lower = pnanovdb_upper_get_child(PNANOVDB_GRID_TYPE_FLOAT, buf, upper, un);
                    pnanovdb_uint32_t ln = pnanovdb_lower_coord_to_offset(&hdda.voxel);
                    if (pnanovdb_lower_get_child_mask(buf, lower, ln)) {
                        pnanovdb_leaf_handle_t leaf = pnanovdb_lower_get_child(PNANOVDB_GRID_TYPE_FLOAT, buf, lower, ln);
                        level = 0;
                        isActive = 1;
                        pnanovdb_coord_t lb = pnanovdb_leaf_get_bbox_min(buf, leaf);
                        pnanovdb_coord_t e8 = pnanovdb_coord_uniform(8);
                        pnanovdb_coord_t lb8 = pnanovdb_coord_add(lb, e8);
                        nmin = pnanovdb_coord_to_vec3(lb);
                        nmax = pnanovdb_coord_to_vec3(lb8);
                    } else {
                        level = 1;
                        isActive = pnanovdb_lower_get_value_mask(buf, lower, ln);
                        pnanovdb_coord_t a = pnanovdb_lower_get_bbox_min(buf, lower);
                        pnanovdb_coord_t b = pnanovdb_lower_get_bbox_max(buf, lower);
                        nmin = pnanovdb_coord_to_vec3(a);
                        nmax = pnanovdb_coord_to_vec3(b);
                    }
                } else {
                    level = 2;
                    isActive = pnanovdb_upper_get_value_mask(buf, upper, un);
                    pnanovdb_coord_t a = pnanovdb_upper_get_bbox_min(buf, upper);
                    pnanovdb_coord_t b = pnanovdb_upper_get_bbox_max(buf, upper);
                    nmin = pnanovdb_coord_to_vec3(a);
                    nmax = pnanovdb_coord_to_vec3(b);
                }
            } else {
                level = 3;
                isActive = pnanovdb_root_tile_get_state(buf, tile) != 0u;
                pnanovdb_coord_t a = pnanovdb_root_get_bbox_min(buf, accessor.root);
                pnanovdb_coord_t b = pnanovdb_root_get_bbox_max(buf, accessor.root);
                nmin = pnanovdb_coord_to_vec3(a);
                nmax = pnanovdb_coord_to_vec3(b);
            }
        } else {
            isActive = pnanovdb_readaccessor_is_active(PNANOVDB_GRID_TYPE_FLOAT, buf, &accessor, &hdda.voxel);
            pnanovdb_coord_t v1 = pnanovdb_coord_add(hdda.voxel, one);
            nmin = pnanovdb_coord_to_vec3(hdda.voxel);
            nmax = pnanovdb_coord_to_vec3(v1);
        }
        out_voxel[3 * visits] = hdda.voxel.x;
        out_voxel[3 * visits + 1] = hdda.voxel.y;
        out_voxel[3 * visits + 2] = hdda.voxel.z;
        out_dim[visits] = hdda.dim;
        out_active[visits] = (uint8_t)isActive;
        out_level[visits] = level;
        float tMinNode = 0.0f, tMaxNode = 1e10f;
        if (isActive) {
            out_box[6 * visits] = nmin.x; out_box[6 * visits + 1] = nmin.y; out_box[6 * visits + 2] = nmin.z;
            out_box[6 * visits + 3] = nmax.x; out_box[6 * visits + 4] = nmax.y; out_box[6 * visits + 5] = nmax.z;
            pnanovdb_hdda_ray_clip(&nmin, &nmax, &origin, &tMinNode, &direction, &tMaxNode);
        } else {
            for (int k = 0; k < 6; k++) out_box[6 * visits + k] = 0.0f;
        }
        float nx = hdda.next.x < hdda.next.y ? hdda.next.x : hdda.next.y;
        nx = nx < hdda.next.z ? nx : hdda.next.z;
        out_t[3 * visits] = hdda.tmin;
        out_t[3 * visits + 1] = nx;
        out_t[3 * visits + 2] = tMinNode;
        visits++;
    }
    return visits;
}
