// ref_cpp_shim.h - the few glm / sgl / Vulkan declarations that the reference's C++ supervoxel and
// density-field sources (src/PathTracer/SuperVoxelGrid.cpp, src/DensityField.cpp) use, so that they
// compile unmodified for the CPU (TEST INFRASTRUCTURE ONLY; oracle/ref_build.py, outputs in
// oracle/_ref).  glm and sgl are not part of the reference tree; only what these two files touch is
// declared.  Device images become host byte buffers: uploadData keeps a copy that the driver reads.
#pragma once
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace glm {
struct vec2 {
    float x = 0.0f, y = 0.0f;
    vec2() = default;
    vec2(float a, float b) : x(a), y(b) {}
};
struct vec3 {
    float x = 0.0f, y = 0.0f, z = 0.0f;
    vec3() = default;
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
};
struct ivec3 {
    int x = 0, y = 0, z = 0;
    ivec3() = default;
    explicit ivec3(int s) : x(s), y(s), z(s) {}
    ivec3(int a, int b, int c) : x(a), y(b), z(c) {}
};
// glm::clamp(x, lo, hi) = min(max(x, lo), hi)
inline float clamp(float x, float lo, float hi) { return std::min(std::max(x, lo), hi); }
}  // namespace glm

namespace sgl {
// integer division rounded up
inline int iceil(int x, int y) { return (x + y - 1) / y; }

class Logfile {
public:
    static Logfile* get() {
        static Logfile l;
        return &l;
    }
    void throwError(const std::string& msg, bool = true) { throw std::runtime_error(msg); }
    void writeError(const std::string&, bool = true) {}
    void writeInfo(const std::string&) {}
};

// min and max of an array (the initial pair is the identity of the reduction)
inline std::pair<float, float> reduceFloatArrayMinMax(
        const float* values, size_t n,
        std::pair<float, float> init = {std::numeric_limits<float>::max(), std::numeric_limits<float>::lowest()}) {
    for (size_t i = 0; i < n; i++) {
        init.first = std::min(init.first, values[i]);
        init.second = std::max(init.second, values[i]);
    }
    return init;
}
inline std::pair<float, float> reduceUnormByteArrayMinMax(const uint8_t* values, size_t n) {
    std::pair<float, float> r = {1.0f, 0.0f};
    for (size_t i = 0; i < n; i++) {
        r.first = std::min(r.first, float(values[i]) / 255.0f);
        r.second = std::max(r.second, float(values[i]) / 255.0f);
    }
    return r;
}
inline std::pair<float, float> reduceUnormShortArrayMinMax(const uint16_t* values, size_t n) {
    std::pair<float, float> r = {1.0f, 0.0f};
    for (size_t i = 0; i < n; i++) {
        r.first = std::min(r.first, float(values[i]) / 65535.0f);
        r.second = std::max(r.second, float(values[i]) / 65535.0f);
    }
    return r;
}
}  // namespace sgl

// IEEE half: only its use as storage is declared (the float paths are what the oracle exercises)
class HalfFloat {
public:
    HalfFloat() = default;
    explicit HalfFloat(float v) : f(v) {}
    explicit operator float() const { return f; }

private:
    float f = 0.0f;
};
namespace sgl {
inline std::pair<float, float> reduceHalfFloatArrayMinMax(const HalfFloat* values, size_t n) {
    std::pair<float, float> r = {std::numeric_limits<float>::max(), std::numeric_limits<float>::lowest()};
    for (size_t i = 0; i < n; i++) {
        r.first = std::min(r.first, float(values[i]));
        r.second = std::max(r.second, float(values[i]));
    }
    return r;
}
}  // namespace sgl

enum class ScalarDataFormat { FLOAT, BYTE, SHORT, FLOAT16 };

// RenderSettings.hpp:51-55
enum class GridInterpolationType { NEAREST, STOCHASTIC, TRILINEAR };

typedef int VkFormat;
enum : int {
    VK_FORMAT_UNDEFINED = 0, VK_FORMAT_R8_UNORM = 9, VK_FORMAT_R8_UINT = 13, VK_FORMAT_R16_UNORM = 70,
    VK_FORMAT_R16_SFLOAT = 76, VK_FORMAT_R32_SFLOAT = 100, VK_FORMAT_R32G32_SFLOAT = 103,
    VK_IMAGE_TYPE_3D = 2, VK_IMAGE_USAGE_TRANSFER_DST_BIT = 2, VK_IMAGE_USAGE_SAMPLED_BIT = 4,
    VK_SAMPLER_ADDRESS_MODE_CLAMP_TO_BORDER = 3, VK_BORDER_COLOR_FLOAT_TRANSPARENT_BLACK = 0,
    VK_BORDER_COLOR_INT_TRANSPARENT_BLACK = 1, VK_FILTER_NEAREST = 0
};

namespace sgl {
namespace vk {
class Device {};
struct ImageSettings {
    uint32_t width = 1, height = 1, depth = 1;
    int imageType = 0, usage = 0, format = 0;
};
struct ImageSamplerSettings {
    int addressModeU = 0, addressModeV = 0, addressModeW = 0, borderColor = 0, minFilter = 0, magFilter = 0;
};
class Image {
public:
    void uploadData(size_t size, const void* data) {
        bytes.resize(size);
        memcpy(bytes.data(), data, size);
    }
    std::vector<uint8_t> bytes;
};
class Texture {
public:
    Texture(Device*, const ImageSettings& s, const ImageSamplerSettings&) : settings(s), image(new Image) {}
    std::shared_ptr<Image> getImage() { return image; }
    ImageSettings settings;
    std::shared_ptr<Image> image;
};
typedef std::shared_ptr<Texture> TexturePtr;
}  // namespace vk
}  // namespace sgl
