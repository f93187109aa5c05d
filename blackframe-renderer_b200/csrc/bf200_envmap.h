// Environment-map light: a packet-bound, piecewise-constant latitude-longitude map importance-
// sampled by texel (EnvironmentLights.hpp:468-1075, EnvironmentMapLightT<float>).
//
// This header holds the host construction of the sampling tables, which runs in float exactly as
// the reference's create() does (EnvironmentLights.hpp:470-733), the power() evaluation
// (:853-885), and the device view that the batch kernels of bf200_envmap.cu read. The oracle
// links the construction as well; its sampling and lookups are restated separately on the CPU.
#pragma once

#include <cstdint>
#include <vector>

namespace bf200 {

// The model after create(). Matrices are the rotation's upper 3x3 (row-major) of the 4x4 built by
// rotation_matrix (Quaternion.hpp:118-150) and of its Gauss-Jordan inverse (MatrixOperations.hpp:
// 31-94): vectors are transformed with them only.
struct EnvironmentTables {
    uint32_t width = 0;
    uint32_t height = 0;
    std::vector<float> texels;       // width * height * 4 lanes, row-major, row 0 at local +Y
    float nanometers[4] = {};        // the packet the map is bound to
    float quaternion[4] = {};        // environment-to-world rotation x, y, z, w
    float matrix[9] = {};            // environment to world
    float inverse[9] = {};           // world to environment
    std::vector<float> azimuth;      // width + 1 boundaries, 0 .. 2 pi
    std::vector<float> cosine;       // height + 1 boundaries, 1 .. -1
    std::vector<float> row_cdf;      // height
    std::vector<float> column_cdfs;  // width * height, one conditional CDF per row
    std::vector<float> density;      // width * height solid-angle densities
    float lane_peak[4] = {};
    float lane_integral[4] = {};     // normalized solid-angle integral per lane
    bool black = true;
};

// Codes of a failed construction or power() call: the reference's StatusCode.
enum EnvironmentError : int {
    kEnvironmentOk = 0,
    kEnvironmentInvalid = 1,    // invalid_argument
    kEnvironmentExhausted = 2,  // resource_exhausted
};

// create(width, height, texels, wavelengths, environment_to_world). texels: width * height
// records of 4 lanes. quaternion: x, y, z, w. Returns kEnvironmentOk, or a code with the
// reference's message in `message`.
int build_environment_tables(uint32_t width, uint32_t height, const float* texels, const float nanometers[4],
                             const float quaternion[4], EnvironmentTables& out, const char*& message);

// power(scene_bounds): the per-lane power of the map over the bounding sphere of [lo, hi]; `out`
// is left as it is when the call fails.
int environment_power(const EnvironmentTables& t, const float lo[3], const float hi[3], float out[4],
                      const char*& message);

// Per-query status codes of the batch kernels (0: the reference returns a value).
enum EnvironmentQueryStatus : uint32_t {
    kEnvQueryOk = 0,
    kEnvQueryInvalidSample = 1,     // canonical sample outside [0, 1)^2
    kEnvQueryInvalidDirection = 2,  // not a finite unit (pdf) / representable non-zero (le) direction
    kEnvQueryEscaped = 3,           // a lookup escaped its angular partition or CDF
    kEnvQueryUnstable = 4,          // rotation cannot keep the selected texel
    kEnvQueryNotRepresentable = 5,  // an interior sample or the resulting direction is not representable
};

// Device view of the tables (device pointers).
struct EnvironmentView {
    uint32_t width;
    uint32_t height;
    const float* texels;
    const float* azimuth;
    const float* cosine;
    const float* row_cdf;
    const float* column_cdfs;
    const float* density;
    float matrix[9];
    float inverse[9];
    uint32_t black;
};

}  // namespace bf200
