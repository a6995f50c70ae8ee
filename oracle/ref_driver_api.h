// ref_driver_api.h - state shared by the reference-shader variants (TEST INFRASTRUCTURE ONLY).
#pragma once
#include "ref_shim.h"

namespace glslref {
struct RefState {
    Parameters params;
    FrameInfo frame;
    sampler3D grid;       // gridImage
    sampler3D gradient;   // gradientImage (ISOSURFACE_TYPE_GRADIENT variants)
    sampler3D emission;   // emissionImage (USE_EMISSION variants)
    sampler1DArray tf;    // transferFunctionTexture (USE_TRANSFER_FUNCTION variants)
    sampler3D sv;         // superVoxelGridImage (RG32F)
    usampler3D svocc;     // superVoxelGridOccupancyImage
    sampler2D env;        // environmentMapTexture
    sampler2D envocta;    // environmentMapOctahedralTexture (mip chain)
    uimage3D occ;         // occupancyGridImage
    image2D result, acc;  // resultImage, accImage
    image2D dblend, dnear;  // depthBlendedImage, depthNearestOpaqueImage (WRITE_DEPTH_*_MAP variants)
    image2D firstw, flow, flowrev, reproj;  // firstW, flowImage, flowReverseImage, reprojUVImage
    image2D normal, dnabla, dfwidth;        // normalImage, depthNablaImage, depthFwidthImage
    Light lights[16];     // LightsBuffer
};
extern RefState g_ref;
extern thread_local uvec3 gl_global_invocation_id;
extern uint ref_seed_offset;
}  // namespace glslref

struct RefVariant {
    const char* name;
    void (*run_pixel)(int x, int y);
};
extern const RefVariant ref_variants[];
extern const int ref_num_variants;
