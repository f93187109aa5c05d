// Host checks of scene records, shared by scene creation (bf200_host.cu), the mesh importers
// (bf200_import.cpp), the environment map (bf200_envmap.cpp) and the scene JSON codec
// (bf200_scene_json.cpp). Each restates the create() of the reference record it names, so every
// entry point refuses exactly what the reference refuses.
#pragma once

#include <cstdint>

#include "bf200.h"

namespace bf200 {

constexpr uint32_t kClosureCapacity = 8U;  // MaximumClosureCount (ClosureSet.hpp:15)

// ClosureSet::append_* and the closure models' create() (ClosureSet.hpp:76-260,
// ClosureMixture.hpp:340-480): weights in [0, 1], the parameters each kind takes (and zeros in
// the rest), the lobes each kind is appended with.
bool valid_closure_payload(const bf200_closure_v1& c);

// The lobes ClosureSet::append_* gives a closure kind (BF200_LOBE_* bits; 0 for an unknown kind).
uint32_t closure_lobes(uint32_t kind);

// build_component_distribution (ClosureMixture.hpp:122-234): the component probabilities of a
// closure mixture projected onto the 2^-24 sampler grid and their CDF; false when they do not
// form a distribution at that precision.
bool project_component_distribution(const float* probabilities, uint32_t n, float* out_p, float* out_cdf);

// unit_direction (PunctualLights.hpp): finite, squared length within 128 ulp of one.
bool unit_direction3(const float* d);

// exact_special_cosine (PunctualLights.hpp:186-197).
float special_cosine(float angle);

// The create() checks of PointLight, DirectionalLight and SpotLight (PunctualLights.hpp:373-388,
// 494-509, 595-650). A spot light's cone cosines are written to cos_inner and cos_outer.
bool punctual_light_checks(const bf200_punctual_light_v1& light, float& cos_inner, float& cos_outer);

// Gauss-Jordan inverse with partial pivoting of a row-major 4x4 float matrix
// (MatrixOperations.hpp:31-94); false for a non-finite input or result or a zero pivot.
bool invert_matrix4(const float (&m)[16], float (&out)[16]);

// The unit-normal check of TriangleMesh::create: finite, squared length within 256 ulp of one.
bool unit_normal(float x, float y, float z);

// TriangleMesh::create (Blackframe/Engine/Source/TriangleMesh.cpp:60-130) over aligned arrays
// (3 positions, 3 normals and 2 texture coordinates per vertex; 3 indices per triangle): null
// when the mesh is valid, else the reference's message for the first check that fails. Counts
// above the 32-bit index domain are the caller's check (resource_exhausted in the reference).
const char* triangle_mesh_problem(const float* positions, const float* normals, const float* uvs,
                                  uint64_t vertices, const uint32_t* triangles, uint64_t triangle_count);

}  // namespace bf200
