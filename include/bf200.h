/*
 * bf200 — B200-native (sm_100a) wavefront path-tracing backend for Blackframe.
 *
 * This header is the whole drop-in boundary. It has three parts:
 *
 *   1. The Blackframe extension ABI v1 and XPU backend ABI v1 (device enumeration). Names,
 *      values and layouts are the ones a Blackframe host binds:
 *        - Blackframe/Extensions/Abi/Include/Blackframe/Extensions/ExtensionAbi.h:6-101
 *        - Blackframe/XPU/BackendAbi/Include/Blackframe/XPU/XpuBackendAbi.h:7-55
 *      The loader resolves `blackframe_query_extension` and asks `get_interface` for an
 *      interface id (Blackframe/XPU/Host/Source/XpuBackend.cpp:57-100).
 *
 *   2. A versioned render interface (BF200_RENDER_INTERFACE_ID_*), returned by the same
 *      `get_interface` call. It replaces the C++ entry point
 *        trace_cuda_wavefront_transport(workspace, CudaSceneSoA, CudaSceneBvh,
 *                                       span<CudaWavefrontPathInput>, LightSampler, options)
 *      (Blackframe/Backends/GPU/CUDA/Include/Blackframe/Backends/GPU/CUDA/
 *       WavefrontTransport.hpp:197-208) and the scene upload / BVH build that precede it
 *      (SceneSoA.hpp:33, SceneBvh.cpp:1109).
 *
 *   3. The same render entry points as plain exported C functions (bf200_*), for FFI callers
 *      (ctypes, cgo, JNI) that do not want to go through the extension table.
 *
 * Conventions follow ExtensionAbi.h: every call returns a blackframe_status, every structure
 * that can grow carries struct_size first, reserved words must be zero, and no C++ type,
 * exception or allocator crosses the boundary. Host pointers are plain host memory; functions
 * with a `_device` suffix take CUDA device pointers instead.
 */
#ifndef BF200_H
#define BF200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__cplusplus)
#define BF200_EXTERN_C extern "C"
#define BF200_NOEXCEPT noexcept
#else
#define BF200_EXTERN_C
#define BF200_NOEXCEPT
#endif

#if defined(__GNUC__) || defined(__clang__)
#define BF200_EXPORT __attribute__((visibility("default")))
#else
#define BF200_EXPORT
#endif

/* ---------------------------------------------------------------------------------------- */
/* 1. Extension ABI v1 (layouts and values mirror ExtensionAbi.h:37-101)                    */
/* ---------------------------------------------------------------------------------------- */

#ifndef BLACKFRAME_EXTENSIONS_EXTENSION_ABI_H
#define BLACKFRAME_EXTENSION_ABI_MAJOR UINT32_C(1)
#define BLACKFRAME_EXTENSION_ABI_MINOR UINT32_C(0)
#define BLACKFRAME_EXTENSION_QUERY_SYMBOL "blackframe_query_extension"

typedef uint32_t blackframe_status;
#define BLACKFRAME_STATUS_SUCCESS ((blackframe_status)0u)
#define BLACKFRAME_STATUS_INVALID_ARGUMENT ((blackframe_status)1u)
#define BLACKFRAME_STATUS_UNSUPPORTED_ABI ((blackframe_status)2u)
#define BLACKFRAME_STATUS_INTERFACE_NOT_FOUND ((blackframe_status)3u)
#define BLACKFRAME_STATUS_INVALID_STATE ((blackframe_status)4u)
#define BLACKFRAME_STATUS_OUT_OF_RANGE ((blackframe_status)5u)
#define BLACKFRAME_STATUS_EXTENSION_FAILURE ((blackframe_status)6u)

typedef struct blackframe_interface_id {
    uint64_t high;
    uint64_t low;
} blackframe_interface_id;

typedef struct blackframe_utf8_view {
    const char* data;
    uint32_t size;
    uint32_t reserved;
} blackframe_utf8_view;

typedef struct blackframe_extension_query_v1 {
    uint32_t struct_size;
    uint32_t abi_major;
    uint32_t abi_minor;
    uint32_t reserved;
} blackframe_extension_query_v1;

typedef blackframe_status (*blackframe_extension_get_interface_fn)(
    void* extension_context, blackframe_interface_id interface_id, uint32_t requested_major,
    uint32_t requested_minor, void* out_interface, uint32_t out_interface_size) BF200_NOEXCEPT;

typedef void (*blackframe_extension_shutdown_fn)(void* extension_context) BF200_NOEXCEPT;

typedef struct blackframe_extension_api_v1 {
    uint32_t struct_size;
    uint32_t abi_major;
    uint32_t abi_minor;
    uint32_t reserved;
    void* extension_context;
    blackframe_extension_get_interface_fn get_interface;
    blackframe_extension_shutdown_fn shutdown;
} blackframe_extension_api_v1;
#endif /* BLACKFRAME_EXTENSIONS_EXTENSION_ABI_H */

/* Replaces ExtensionAbi.h:99-101 — the single symbol a Blackframe host resolves. */
BF200_EXTERN_C BF200_EXPORT blackframe_status
blackframe_query_extension(const blackframe_extension_query_v1* query,
                           blackframe_extension_api_v1* out_extension) BF200_NOEXCEPT;

/* ---------------------------------------------------------------------------------------- */
/* XPU backend ABI v1 (XpuBackendAbi.h:10-55): enumeration only                             */
/* ---------------------------------------------------------------------------------------- */

#ifndef BLACKFRAME_XPU_XPU_BACKEND_ABI_H
#define BLACKFRAME_XPU_BACKEND_ABI_MAJOR UINT32_C(1)
#define BLACKFRAME_XPU_BACKEND_ABI_MINOR UINT32_C(0)
#define BLACKFRAME_XPU_BACKEND_INTERFACE_ID_HIGH UINT64_C(0x96c6e70dd06b4b93)
#define BLACKFRAME_XPU_BACKEND_INTERFACE_ID_LOW UINT64_C(0xa9514ab777f49d37)

typedef uint32_t blackframe_xpu_device_kind;
#define BLACKFRAME_XPU_DEVICE_KIND_UNKNOWN ((blackframe_xpu_device_kind)0u)
#define BLACKFRAME_XPU_DEVICE_KIND_CPU ((blackframe_xpu_device_kind)1u)
#define BLACKFRAME_XPU_DEVICE_KIND_GPU ((blackframe_xpu_device_kind)2u)
#define BLACKFRAME_XPU_DEVICE_KIND_ACCELERATOR ((blackframe_xpu_device_kind)3u)

typedef struct blackframe_xpu_device_descriptor_v1 {
    uint32_t struct_size;
    blackframe_xpu_device_kind kind;
    uint64_t identifier_high;
    uint64_t identifier_low;
    blackframe_utf8_view name;
    blackframe_utf8_view vendor;
    uint64_t reserved[4];
} blackframe_xpu_device_descriptor_v1;

typedef blackframe_status (*blackframe_xpu_get_device_count_fn)(
    void* backend_context, uint32_t* out_device_count) BF200_NOEXCEPT;
typedef blackframe_status (*blackframe_xpu_get_device_descriptor_fn)(
    void* backend_context, uint32_t device_index,
    blackframe_xpu_device_descriptor_v1* out_descriptor) BF200_NOEXCEPT;

typedef struct blackframe_xpu_backend_api_v1 {
    uint32_t struct_size;
    uint32_t abi_major;
    uint32_t abi_minor;
    uint32_t reserved;
    void* backend_context;
    blackframe_utf8_view backend_name;
    blackframe_xpu_get_device_count_fn get_device_count;
    blackframe_xpu_get_device_descriptor_fn get_device_descriptor;
    uint64_t reserved_slots[4];
} blackframe_xpu_backend_api_v1;
#endif /* BLACKFRAME_XPU_XPU_BACKEND_ABI_H */

/* ---------------------------------------------------------------------------------------- */
/* 2. Render interface v1 records                                                           */
/* ---------------------------------------------------------------------------------------- */

#define BF200_RENDER_ABI_MAJOR UINT32_C(1)
#define BF200_RENDER_ABI_MINOR UINT32_C(1)
#define BF200_RENDER_INTERFACE_ID_HIGH UINT64_C(0x6266323030726e64) /* "bf200rnd" */
#define BF200_RENDER_INTERFACE_ID_LOW UINT64_C(0x7761766566726e31) /* "wavefrn1" */

/* Closure kinds: renderer::ClosureKind (Blackframe/Renderer/Include/Blackframe/Renderer/
 * ClosureSet.hpp:15-24). */
#define BF200_CLOSURE_NONE 0u
#define BF200_CLOSURE_LAMBERTIAN_REFLECTION 1u
#define BF200_CLOSURE_ROUGH_DIFFUSE_REFLECTION 2u
#define BF200_CLOSURE_ROUGH_CONDUCTOR_REFLECTION 3u
#define BF200_CLOSURE_ROUGH_DIELECTRIC 4u
#define BF200_CLOSURE_SPECULAR_REFLECTION 5u
#define BF200_CLOSURE_SPECULAR_TRANSMISSION 6u

/* Scattering lobe bits: renderer::ScatteringLobe (TransportConventions.hpp:44-52). */
#define BF200_LOBE_DIFFUSE 0x01u
#define BF200_LOBE_GLOSSY 0x02u
#define BF200_LOBE_SPECULAR 0x04u
#define BF200_LOBE_REFLECTION 0x08u
#define BF200_LOBE_TRANSMISSION 0x10u
#define BF200_LOBE_VOLUME 0x20u

/* Path terminations: renderer::BsdfOnlyPathTermination (BsdfOnlyPathLoop.hpp:84-90). */
#define BF200_TERMINATION_ESCAPED_ENVIRONMENT 0u
#define BF200_TERMINATION_DEPTH_LIMIT 1u
#define BF200_TERMINATION_OUTSIDE_BSDF_SUPPORT 2u
#define BF200_TERMINATION_ZERO_THROUGHPUT 3u
#define BF200_TERMINATION_RUSSIAN_ROULETTE 4u

/* Per-lane failure codes. A lane that fails keeps its last state and reports the first failure;
 * nothing is substituted (the reference's "no fallback" rule, WavefrontTransport.cpp:612-617). */
#define BF200_LANE_OK 0u
#define BF200_LANE_NUMERICAL_FAILURE 1u   /* a checked float operation was not representable */
#define BF200_LANE_UNSUPPORTED 2u         /* the lane reached a feature this backend rejects */
#define BF200_LANE_TRAVERSAL_FAILURE 3u   /* traversal stack overflow / invalid topology */

/* One closure record: renderer::ClosureT (ClosureSet.hpp:45-50), 64 bytes. Parameters follow
 * the reference's packing: conductor eta[0..3], k[4..7], alpha_x[8], alpha_y[9]; dielectric
 * exterior eta[0], interior eta[1], alpha_x[2], alpha_y[3]. */
typedef struct bf200_closure_v1 {
    uint32_t kind;
    uint32_t lobes;
    float weight[4];
    float parameters[10];
} bf200_closure_v1;

/* A material: engine::SceneSpectralMaterial (FrameScene.hpp:158-166) resolved at the frame's
 * single wavelength packet. frame_mode: 0 shading normal, 1 surface tangent
 * (SceneClosureFrameMode, FrameScene.hpp:81-84). */
typedef struct bf200_material_v1 {
    uint32_t material_id;
    uint32_t closure_offset;
    uint32_t closure_count;
    uint32_t frame_mode;
    float tangent_rotation_radians;
    float component_probabilities[8];
    float emitted_radiance[4];
    uint32_t reserved[3];
} bf200_material_v1;

/* Geometry kinds. A sphere (renderer::SphereT, Sphere.hpp:303-437; FrameScene has no analytic
 * primitive, so this kind is an addition) is its centre, the geometry's one vertex
 * (vertex_count = 1, triangle_count = 0), and `radius`, in object space. Its hits are the
 * reference's exact quadratic roots; closest-hit queries report its outward normal in the
 * barycentric words. Emissive spheres are refused (no substitution): lights are meshes. */
#define BF200_GEOMETRY_TRIANGLES 0u
#define BF200_GEOMETRY_SPHERE 1u

typedef struct bf200_geometry_v1 {
    uint32_t geometry_id;
    uint32_t vertex_offset;
    uint32_t vertex_count;
    uint32_t triangle_offset;
    uint32_t triangle_count;
    uint32_t kind;      /* BF200_GEOMETRY_*; 0 for a triangle mesh */
    float radius;       /* spheres; 0 for a triangle mesh */
    uint32_t reserved;
} bf200_geometry_v1;

/* An instance after hierarchy resolution, in the committed (identifier-sorted) order. The
 * matrices are the resolved object_to_world transform and its inverse exactly as FrameScene
 * stores them (row-major 4x4; SceneSoaAbi.hpp columns instance_local_to_world /
 * instance_world_to_local). */
typedef struct bf200_instance_v1 {
    uint32_t instance_id;
    uint32_t object_id;
    uint32_t geometry_index;
    uint32_t material_index;
    uint32_t visibility_mask;
    uint32_t reserved[3];
    float object_to_world[16];
    float world_to_object[16];
} bf200_instance_v1;

/* Punctual lights: engine::ScenePointLight, SceneDirectionalLight and SceneSpotLight
 * (FrameScene.hpp:191-215), sampled as renderer::PointLight, DirectionalLight and SpotLight
 * (PunctualLights.hpp:370-815). spectrum: the point light's spectral radiant intensity, the
 * directional light's spectral irradiance, or the spot light's on-axis spectral radiant intensity,
 * at the frame's packet. direction: the directional light's propagation direction (from the source
 * into the scene) or the spot light's emission direction; unit length. 72 bytes. */
#define BF200_PUNCTUAL_POINT 1u
#define BF200_PUNCTUAL_DIRECTIONAL 2u
#define BF200_PUNCTUAL_SPOT 3u

typedef struct bf200_punctual_light_v1 {
    uint32_t kind;                 /* BF200_PUNCTUAL_* */
    uint32_t reserved;
    float position[3];             /* point and spot */
    float position_error[3];       /* point and spot: absolute world-space position error, >= 0 */
    float direction[3];            /* directional and spot */
    float inner_half_angle;        /* spot, radians: 0 <= inner <= outer < pi, outer > 0 */
    float outer_half_angle;
    float spectrum[4];
} bf200_punctual_light_v1;

/* A committed frame scene (engine::FrameScene, FrameScene.hpp:101-316), flattened. Triangle
 * vertex indices are local to their geometry. The light registry is the punctual lights in the
 * given order, then the mesh area lights, derived exactly as FrameScene derives them
 * (FrameScene.cpp:201-261): one light per instance whose material emits, in instance order.
 * A material may hold up to 8 closures (MaximumClosureCount), sampled by its component
 * probabilities as SceneClosureMixture samples them. A caller built against the layout without
 * `punctual_lights` passes struct_size = BF200_SCENE_DESC_V1_BASE_SIZE and no punctual lights. */
typedef struct bf200_scene_desc_v1 {
    uint32_t struct_size;
    uint32_t geometry_count;
    uint32_t vertex_count;
    uint32_t triangle_count;
    uint32_t material_count;
    uint32_t closure_count;
    uint32_t instance_count;
    uint32_t punctual_light_count; /* entries of punctual_lights */
    const bf200_geometry_v1* geometries;
    const float* positions;        /* 3 * vertex_count */
    const float* normals;          /* 3 * vertex_count */
    const float* texture_coordinates; /* 2 * vertex_count */
    const uint32_t* triangles;     /* 3 * triangle_count */
    const bf200_material_v1* materials;
    const bf200_closure_v1* closures;
    const bf200_instance_v1* instances;
    float wavelength_nanometers[4];
    float wavelength_pdf[4];
    float environment_radiance[4];
    uint32_t reserved[4];
    const bf200_punctual_light_v1* punctual_lights;
} bf200_scene_desc_v1;
#define BF200_SCENE_DESC_V1_BASE_SIZE ((uint32_t)offsetof(bf200_scene_desc_v1, punctual_lights))

/* renderer::Ray (48 bytes, the same size as the reference TransportRay). */
typedef struct bf200_ray_v1 {
    float origin[3];
    float direction[3];
    float t_min;
    float t_max;
    float time;
    uint32_t mask;
    uint32_t medium;
    uint32_t reserved;
} bf200_ray_v1;

/* renderer::SampleStreamIndex (SampleStream.hpp:12-18), 24 bytes. */
typedef struct bf200_sample_index_v1 {
    uint32_t pixel_x;
    uint32_t pixel_y;
    uint64_t sample_index;
    uint64_t seed;
} bf200_sample_index_v1;

/* engine::CudaWavefrontPathInput (WavefrontTransport.hpp:27-32) for a primary path whose
 * initial state is PathState::create_initial (beta 1, no radiance, depth 0, vacuum). */
typedef struct bf200_path_input_v1 {
    bf200_ray_v1 primary_ray;
    bf200_sample_index_v1 sample;
    uint64_t reserved;
} bf200_path_input_v1;

/* engine::CudaWavefrontPathResult (WavefrontTransport.hpp:52-57) flattened. */
typedef struct bf200_path_result_v1 {
    float beta[4];
    float radiance[4];
    uint32_t depth;
    uint32_t depth_counters[5]; /* diffuse, glossy, specular, transmission, volume */
    float eta_scale;
    uint32_t delta_flags;
    uint32_t termination;
    uint32_t blocked_depth_limits;
    uint32_t lane_status;  /* BF200_LANE_* */
    uint32_t segments;     /* extension segments traced by this path */
    bf200_ray_v1 terminal_ray;
} bf200_path_result_v1;

/* engine::CudaWavefrontTransportOptions (WavefrontTransport.hpp:134-142), render subset. */
typedef struct bf200_transport_options_v1 {
    uint32_t struct_size;
    uint32_t mis_heuristic;        /* 0 balance, 1 power (MisHeuristics.hpp:13-16) */
    uint32_t depth_limits[5];      /* diffuse, glossy, specular, transmission, volume */
    uint32_t roulette_enabled;
    uint32_t roulette_first_eligible_depth;
    float roulette_minimum_survival;
    float roulette_maximum_survival;
    uint32_t instrumentation; /* 1: time every stage with CUDA events (CudaWavefrontInstrumentationMode::nsight) */
    uint32_t sampler;         /* BF200_SAMPLER_*: 0 hash SampleStream (reference parity), 1 Owen-scrambled Sobol */
    uint32_t reserved[3];
} bf200_transport_options_v1;

/* Transport samplers. BF200_SAMPLER_HASH draws SampleStream::indexed_bits (SampleStream.hpp:31-67)
 * exactly as the reference transport does. BF200_SAMPLER_OWEN_SOBOL draws the Owen-scrambled Sobol
 * coordinate owen_scrambled_sobol_bits(index, d') (OwenScrambling.hpp:11-22) of the same sample
 * index, where d' = 0 and 1 for the two camera-raster dimensions and d + 2 for every other sample
 * dimension d. No reference transport uses Sobol, so this mapping has no reference counterpart;
 * it supports total path depths up to 255. */
#define BF200_SAMPLER_HASH 0u
#define BF200_SAMPLER_OWEN_SOBOL 1u

/* Pinhole camera (PinholeCamera.hpp:52-306) with the host-side constants already derived:
 * half_height = tan(fov/2), half_width = half_height * width/height. */
typedef struct bf200_camera_v1 {
    float origin[3];
    float tangent[3];
    float bitangent[3];
    float normal[3];
    float half_width;
    float half_height;
    float t_min;
    float t_max;
    float time;
    uint32_t mask;
    uint32_t width;
    uint32_t height;
    uint32_t jitter_mode; /* 0 pixel centre, 1 uniform jitter (PixelJitter.hpp:15-18) */
    uint32_t reserved;
} bf200_camera_v1;

/* CIE 1931 sensor constants of the frame's packet (Cie1931Sensor.cpp): per lane the XYZ
 * colour-matching response at the lane wavelength and the lane wavelength pdf, plus the
 * normalisation (1/4)/Y-integral. */
typedef struct bf200_sensor_v1 {
    float response_xyz[4][3];
    float wavelength_pdf[4];
    float normalization;
    uint32_t reserved[3];
} bf200_sensor_v1;

/* A film request: W x H pixels, samples [first_sample, first_sample + samples_per_pixel).
 * Every (pixel, sample) path is traced and added to the film in sample order, exactly as a
 * caller that loops over samples and calls Film::add_sample(x, y, rgb, 1) would. */
typedef struct bf200_film_request_v1 {
    uint32_t struct_size;
    uint32_t samples_per_pixel;
    uint64_t first_sample;
    uint64_t seed;
    uint32_t precision;        /* 0 float32 film (renderer::Film), 1 float64 Neumaier film */
    uint32_t reserved[3];
} bf200_film_request_v1;

/* Film storage. float32: 4 floats per pixel (r, g, b, weight) + count. float64: 8 doubles per
 * pixel (sum r,g,b, weight; compensation r,g,b, weight) + count. */
typedef struct bf200_film_v1 {
    uint32_t width;
    uint32_t height;
    uint32_t precision;
    uint32_t reserved;
    void* sums;            /* host or device pointer, see each call */
    uint64_t* sample_counts;
} bf200_film_v1;

/* engine::CudaWavefrontTransportReport (WavefrontTransport.hpp:97-125), counting subset.
 * terminated_paths counts the paths that finished without a lane failure (every call but
 * bf200_trace_paths_device_noalloc, which leaves it zero). closure_samples,
 * light_samples (the shade stage's WavefrontShadeDetailClosureSampled / LightSampled lanes),
 * miss_segments and continuation_segments are counted by the traces that carry ray cones
 * (bf200_trace_paths_with_cones*), the reference-facing path; other calls leave them zero, so
 * their shading kernels carry no extra counters. */
typedef struct bf200_report_v1 {
    uint32_t struct_size;
    uint32_t registered_light_count;
    uint64_t path_count;
    uint64_t extension_segments;
    uint64_t shadow_segments;
    uint64_t closure_samples;
    uint64_t light_samples;
    uint64_t terminated_paths;
    uint64_t failed_lanes;
    uint32_t first_failure_status;
    uint32_t first_failure_path;
    uint64_t kernel_launches;
    double gpu_milliseconds;
    /* with instrumentation: summed GPU time of each stage, and the iteration count. intersect:
     * closest-hit traversal; shade: routing, the per-closure shading kernels and the shadow-queue
     * compaction; occlude: shadow rays; regenerate: path retirement and camera-ray generation */
    double intersect_milliseconds;
    double shade_milliseconds;
    double occlude_milliseconds;
    double film_milliseconds;
    uint64_t iterations;
    double regenerate_milliseconds;
    /* the reference's stage-lane counts (CudaWavefrontStageLaneCounts, WavefrontTransport.hpp:59-70):
     * extension segments that missed every surface, and paths that continued after shading */
    uint64_t miss_segments;
    uint64_t continuation_segments;
} bf200_report_v1;

typedef struct bf200_context bf200_context;
typedef struct bf200_scene bf200_scene;

/* ---------------------------------------------------------------------------------------- */
/* 3. Exported render entry points                                                          */
/* ---------------------------------------------------------------------------------------- */

/* Creates a context on one CUDA device. Replaces CudaWavefrontTransportWorkspace::create
 * (WavefrontTransport.hpp:160-164): the context owns every device buffer; path capacity is the
 * number of paths kept in flight per wavefront (0 picks the default). */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_context_create(int32_t device_ordinal,
                                                                    uint64_t path_capacity,
                                                                    bf200_context** out_context)
    BF200_NOEXCEPT;
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_context_destroy(bf200_context* context)
    BF200_NOEXCEPT;
/* Device memory the context holds: its wavefront arena and the grow-only workspaces of the film,
 * batch, cone and adjoint calls, in bytes (not its scenes). Replaces
 * CudaWavefrontTransportWorkspace::device_size_bytes (WavefrontTransport.hpp:166). */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_context_device_bytes(const bf200_context* context,
                                                                          uint64_t* out_bytes) BF200_NOEXCEPT;
/* Last error text of a context (UTF-8, owned by the context, valid until the next call). */
BF200_EXTERN_C BF200_EXPORT const char* bf200_context_last_error(const bf200_context* context)
    BF200_NOEXCEPT;

/* Validates and uploads a committed scene, derives the mesh-light registry and builds the
 * BLAS/TLAS on the device. Replaces CudaSceneSoA::upload (SceneSoA.hpp:33) followed by
 * CudaSceneBvh::build (SceneBvh.cpp:1109). */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_scene_create(bf200_context* context,
                                                                  const bf200_scene_desc_v1* desc,
                                                                  bf200_scene** out_scene)
    BF200_NOEXCEPT;
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_scene_destroy(bf200_scene* scene)
    BF200_NOEXCEPT;

/* Traces a batch of primary paths from host inputs to host results (one-sample NEE with
 * balance/power MIS, uniform light selection, Russian roulette). Replaces
 * trace_cuda_wavefront_transport (WavefrontTransport.hpp:197-208). */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_trace_paths(
    bf200_context* context, const bf200_scene* scene, const bf200_path_input_v1* inputs,
    uint64_t path_count, const bf200_transport_options_v1* options,
    bf200_path_result_v1* results, bf200_report_v1* report) BF200_NOEXCEPT;

/* renderer::RayCone (RayCone.hpp:160-189): the cone's radius at the ray origin and its radial
 * slope, 8 bytes (the reference's WavefrontRayCone). */
typedef struct bf200_ray_cone_v1 {
    float width;
    float spread;
} bf200_ray_cone_v1;

/* A depth-zero path state: PathState's throughput, accumulated radiance and eta scale
 * (PathState.hpp:79-160) for a path that starts with depth 0, no delta history and the vacuum
 * medium. 48 bytes. PathState::create_initial is beta 1, radiance 0, eta scale 1. */
typedef struct bf200_path_state_v1 {
    float beta[4];
    float radiance[4];
    float eta_scale;
    uint32_t reserved[3];
} bf200_path_state_v1;

/* bf200_trace_paths with the rest of CudaWavefrontPathInput: every path's ray cone and,
 * optionally, its depth-zero initial state (WavefrontTransport.hpp:27-32). Primary cones go in,
 * and CudaWavefrontTransportBatch::terminal_cones come out (WavefrontTransport.hpp:127-132).
 * - The cone advances to every hit and is re-spread by the selected closure at every scattering
 *   event (CudaWavefrontStages.cu:2832-2870, 3675-3781).
 * - terminal_cones[i] is the cone at results[i].terminal_ray's origin.
 * - initial_states may be null: every path then starts from PathState::create_initial.
 * - The whole call is refused with INVALID_ARGUMENT when a primary cone is not finite and
 *   non-negative, or an initial state has a non-finite or negative spectrum, an eta scale that is
 *   not finite and positive, or a non-zero reserved word (WavefrontTransport.cpp:524-566).
 * - A cone that becomes unrepresentable fails its lane with BF200_LANE_NUMERICAL_FAILURE, as the
 *   reference's shade stage does.
 * Path results are identical to bf200_trace_paths for every lane that starts from the initial
 * state and does not fail. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_trace_paths_with_cones(
    bf200_context* context, const bf200_scene* scene, const bf200_path_input_v1* inputs,
    const bf200_path_state_v1* initial_states, const bf200_ray_cone_v1* primary_cones, uint64_t path_count,
    const bf200_transport_options_v1* options, bf200_path_result_v1* results, bf200_ray_cone_v1* terminal_cones,
    bf200_report_v1* report) BF200_NOEXCEPT;
/* The same with every array in device memory. An invalid primary cone or initial state fails its
 * lane instead of the call (the camera stage's checks, CudaWavefrontStages.cu:1378-1380). */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_trace_paths_with_cones_device(
    bf200_context* context, const bf200_scene* scene, const bf200_path_input_v1* device_inputs,
    const bf200_path_state_v1* device_initial_states, const bf200_ray_cone_v1* device_primary_cones,
    uint64_t path_count, const bf200_transport_options_v1* options, bf200_path_result_v1* device_results,
    bf200_ray_cone_v1* device_terminal_cones, bf200_report_v1* report) BF200_NOEXCEPT;

/* Same as bf200_trace_paths with inputs and results in device memory. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_trace_paths_device(
    bf200_context* context, const bf200_scene* scene, const bf200_path_input_v1* device_inputs,
    uint64_t path_count, const bf200_transport_options_v1* options,
    bf200_path_result_v1* device_results, bf200_report_v1* report) BF200_NOEXCEPT;

/* Allocation-free variant of bf200_trace_paths_device. It has no counterpart in the reference.
 *
 * Why: the ordinary entry point sizes its wavefront arena on first use with cudaMalloc and
 * cudaMallocHost. Some callers cannot let a trace allocate:
 *   - a renderer that has committed the device's memory to its own pools before the first frame,
 *     where a late allocation can fail with out-of-memory halfway through a frame;
 *   - a host that keeps other streams busy, where cudaFree and, often, cudaMalloc synchronise the
 *     whole device and stall unrelated work;
 *   - an interactive loop that cannot absorb the allocator's unpredictable host latency.
 * This call uses a fixed scratch array compiled into the library: a file-scope __device__ array of
 * BF200_NOALLOC_SCRATCH_BYTES, holding at most BF200_NOALLOC_MAX_SLOTS path slots. It makes no
 * cudaMalloc, cudaMallocHost, cudaFree, event or stream creation, or other allocating call. It
 * clears the slot states and counters it needs with cudaMemsetAsync on the context's stream, and
 * reads its per-iteration counters back into host stack memory.
 *
 * path_capacity: slots kept in flight, 0 = BF200_NOALLOC_MAX_SLOTS. A larger value is refused with
 * BLACKFRAME_STATUS_OUT_OF_RANGE. Any path_count is accepted, because finished slots are refilled.
 * Results are identical to bf200_trace_paths_device for the same inputs.
 *
 * The device address of the scratch array is looked up once per device with
 * cudaGetSymbolAddress, at the first call on that device. That first call can also make the CUDA
 * driver load the library's device code, so make it during setup, before any stream capture
 * begins. With BF200_SAMPLER_OWEN_SOBOL, the first call on a device (of this or any other entry
 * point) also fills the library's static Sobol direction table with one blocking
 * cudaMemcpyToSymbol (no allocation, but a synchronous host-to-device copy): make one such call
 * during setup as well if later calls must not block. All calls on one device share the one scratch array: calls that overlap in time, from
 * any context or thread, race and corrupt each other's results, so the caller must serialise
 * them. instrumentation is ignored (no events); the report's timing fields are zero. */
#define BF200_NOALLOC_SCRATCH_BYTES (16u << 20)
#define BF200_NOALLOC_MAX_SLOTS 65536u
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_trace_paths_device_noalloc(
    bf200_context* context, const bf200_scene* scene, const bf200_path_input_v1* device_inputs,
    uint64_t path_count, const bf200_transport_options_v1* options,
    bf200_path_result_v1* device_results, uint32_t path_capacity,
    bf200_report_v1* report) BF200_NOEXCEPT;

/* Renders pinhole-camera paths on the device (camera rays, transport and film accumulation all
 * on the GPU) and adds them to a host film. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_render_film(
    bf200_context* context, const bf200_scene* scene, const bf200_camera_v1* camera,
    const bf200_sensor_v1* sensor, const bf200_film_request_v1* request,
    const bf200_transport_options_v1* options, bf200_film_v1* host_film,
    bf200_report_v1* report) BF200_NOEXCEPT;

/* Same as bf200_render_film with the film in device memory (sums and counts device pointers). */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_render_film_device(
    bf200_context* context, const bf200_scene* scene, const bf200_camera_v1* camera,
    const bf200_sensor_v1* sensor, const bf200_film_request_v1* request,
    const bf200_transport_options_v1* options, bf200_film_v1* device_film,
    bf200_report_v1* report) BF200_NOEXCEPT;

/* One film of a batch: the arguments of one bf200_render_film_device call. */
typedef struct bf200_film_job_v1 {
    uint32_t struct_size;
    uint32_t reserved;
    const bf200_scene* scene;
    const bf200_camera_v1* camera;
    const bf200_sensor_v1* sensor;
    const bf200_film_request_v1* request;
    const bf200_transport_options_v1* options;
    bf200_film_v1* film;      /* device film of this job */
    bf200_report_v1* report;  /* optional */
} bf200_film_job_v1;

/* Renders many films, of any scenes of the context, in one call: the batch rendering the
 * reference's benchmark plan asks of a new backend (many scenes and views of uneven size). Every
 * job's film equals, bit for bit, the film of a bf200_render_film_device call with the same
 * arguments. Jobs run concurrently in `lanes` wavefront lanes (0: chosen from the jobs' path
 * counts and the context's path capacity): each lane has its own CUDA stream, a slice of the
 * path slots and its own radiance buffer, and the host keeps every lane busy without waiting
 * on any single one. Jobs must not share a film (their accumulation order across jobs would be
 * unspecified). Reports carry counts, not stage timings. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_render_films_device(bf200_context* context,
                                                                        const bf200_film_job_v1* jobs,
                                                                        uint32_t job_count, uint32_t lanes)
    BF200_NOEXCEPT;

/* The lane count the context's last bf200_render_films_device call used. With lanes = 0 the count is
 * chosen by measurement: the context keeps the fastest of 2, 4 and 8 lanes per job-size class (the
 * binary order of magnitude of the median job's paths), measuring a new class on the batch's own
 * first jobs (dealt round-robin into three groups of at least eight jobs, one per count, each timed to
 * its drain) when the
 * batch holds at least four such groups, and using a closed-form estimate otherwise. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_context_batch_lanes(const bf200_context* context,
                                                                       uint32_t* lanes) BF200_NOEXCEPT;

/* Path-replay adjoint (the reference has no differentiation; its benchmark plan asks a new backend
 * for an adjoint of the film render). One call renders the film, compares the image with a target
 * and returns the gradient of the loss
 *     loss = sum over pixels and rgb channels of (image - target)^2,  image = film rgb / film weight,
 * with respect to every material's closure weight (per packet lane), the GGX roughness alpha_x and
 * alpha_y of conductor and dielectric closures, and a common factor k on every emitter's radiance
 * (at k = 1; the constant environment is not scaled).
 *
 * Method: the paths are traced once forward into the film, then replayed with the same sample
 * indices. The replay knows each path's final radiance, so a vertex's share of the gradient is what
 * the path adds after it (path replay backpropagation, without a reverse pass). With the sampled
 * directions held fixed, every contribution is linear in the closure weights and the emission, so
 * those gradients are the exact derivatives of this render's loss (finite differences on the same
 * samples agree). Sampling densities, MIS weights and Russian-roulette decisions are held fixed:
 * the roughness gradient is the "detached" estimator, unbiased for the derivative of the expected
 * loss but not equal per sample to a finite difference, and Russian roulette should be off when
 * the weight gradients are compared with finite differences.
 *
 * The film (device, as in bf200_render_film_device) is cleared and holds this call's render on
 * return. The loss and the gradients are summed in float64 by atomics in no fixed order, so their
 * last bits vary between calls. At most 64 materials. The report counts the forward render. */
typedef struct bf200_material_gradient_v1 {
    double weight[4];     /* dLoss / d(closure weight of packet lane l) */
    double roughness[2];  /* dLoss / d(alpha_x), dLoss / d(alpha_y); 0 for Lambert */
    double reserved[2];
} bf200_material_gradient_v1;

typedef struct bf200_adjoint_v1 {
    uint32_t struct_size;
    uint32_t reserved;
    const float* target;                   /* device: height x width x 3 floats, rgb, row-major */
    bf200_material_gradient_v1* gradients; /* device: one record per scene material */
    double* emission_gradient;             /* device: one double, dLoss/dk */
    double loss;                           /* out */
} bf200_adjoint_v1;

BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_render_adjoint_device(
    bf200_context* context, const bf200_scene* scene, const bf200_camera_v1* camera,
    const bf200_sensor_v1* sensor, const bf200_film_request_v1* request,
    const bf200_transport_options_v1* options, bf200_film_v1* film, bf200_adjoint_v1* adjoint,
    bf200_report_v1* report) BF200_NOEXCEPT;

/* The same adjoint as a forward/backward pair for any image loss. The forward is
 * bf200_render_film_device. The caller computes dLoss/d(image) (device, height x width x 3 floats,
 * image = film rgb / film weight) and passes it here with the forward's film (its weights) and
 * arguments. The backward traces every path again to recover its radiance (path vertices are
 * recomputed, not stored, so memory stays bounded by one film chunk), then replays it. It costs
 * about two forward renders; the report counts the re-trace. Gradients as described above. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_render_backward_device(
    bf200_context* context, const bf200_scene* scene, const bf200_camera_v1* camera,
    const bf200_sensor_v1* sensor, const bf200_film_request_v1* request,
    const bf200_transport_options_v1* options, const bf200_film_v1* film, const float* image_adjoint,
    bf200_material_gradient_v1* gradients, double* emission_gradient, bf200_report_v1* report) BF200_NOEXCEPT;

/* Scene upload from the reference's scene SoA blob, ABI v4 (SceneSoaHeader + 194 columns,
 * Blackframe/XPU/Shared/Include/Blackframe/XPU/Shared/SceneSoaAbi.hpp, as CudaSceneSoA::upload
 * serialises a FrameScene; replaces SceneSoA.hpp:33): the header is validated as
 * validate_scene_soa_header does and the FNV-1a content hash is checked; then the scene is created
 * as bf200_scene_create creates it. Punctual lights, normal/bump maps and materials resolved at
 * different wavelength packets are refused with INVALID_STATE (no substitution). On failure
 * `message` (when given) receives the reason. Host memory; the blob is not retained. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_scene_create_from_soa(bf200_context* context,
                                                                           const void* blob, uint64_t size,
                                                                           bf200_scene** scene, char* message,
                                                                           uint64_t message_capacity) BF200_NOEXCEPT;

/* Transform-only refit (engine::AccelBackend::refit, AccelBackend.hpp:55-86): `desc` must be the
 * scene's description with nothing but instance transforms (object_to_world and world_to_object)
 * changed; anything else is refused with INVALID_STATE and never turned into a rebuild. The
 * instance level (matrices, world boxes, the TLAS boxes on its existing topology), the mesh lights
 * and the world normals are recomputed in place; the BLASes are kept. Hits after a refit equal
 * those of a scene created from `desc`. Must not run while a trace of this scene is in flight. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_scene_refit(bf200_scene* scene, const bf200_scene_desc_v1* desc)
    BF200_NOEXCEPT;

/* Power-weighted light selection (LightSampler::create_power_weighted, LightSampler.hpp:110-113;
 * the reference CUDA backend refuses it, WavefrontTransport.cpp:612-617). `spectral_powers` holds
 * the caller's four-lane spectral flux of every scene light in registry order (mesh lights in
 * instance order). Each light's weight is the compensated sum of its lanes over the largest lane
 * of all lights, and the CDF is built from compensated prefix sums, as the reference builds it
 * (bit for bit). Selection and the MIS probability of a light then follow that CDF. A null
 * `spectral_powers` restores uniform selection. Must not run while a trace of the scene is in
 * flight. bf200_light_power_cdf computes the light_count + 1 boundaries alone (host only). */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_scene_set_light_powers(bf200_scene* scene,
                                                                            const float* spectral_powers,
                                                                            uint32_t light_count) BF200_NOEXCEPT;
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_light_power_cdf(const float* spectral_powers,
                                                                     uint32_t light_count, float* boundaries)
    BF200_NOEXCEPT;

/* One light of a spatial light tree: LightTreeInput (LightSampler.hpp:19-25), its conservative
 * world bounds (min <= max, no NaN; +-infinity on every axis for an unbounded light) and its
 * four-lane spectral power, in registry order. 40 bytes. */
typedef struct bf200_light_tree_input_v1 {
    float bounds_min[3];
    float bounds_max[3];
    float spectral_power[4];
} bf200_light_tree_input_v1;

/* LightSampler::create_spatial_tree (LightSampler.cpp:626-951) and its selection at query points
 * (sample(context, u), LightSampler.cpp:1058-1129), bit for bit: for every query the selected slot
 * and its discrete probability, or 0xFFFFFFFF and -1 where the reference refuses that query. A
 * tree the reference refuses to build fails the call (INVALID_ARGUMENT for invalid inputs,
 * OUT_OF_RANGE for unrepresentable powers or bounds). positions: 3 floats per query. Host
 * computation; transport does not select by tree yet. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_light_tree_select(const bf200_light_tree_input_v1* lights,
                                                                      uint32_t light_count, const float* positions,
                                                                      const float* samples, uint64_t query_count,
                                                                      uint32_t* light_indices,
                                                                      float* probabilities) BF200_NOEXCEPT;
/* Selects the scene's lights by the spatial light tree of `lights` (one per scene light, registry
 * order) in every later trace and render: next-event estimation draws a light with
 * LightSampler::sample(context, u) at the shading point, and the MIS weight of an emissive hit
 * uses probability(context, i) at the previous vertex (SceneMisPathLoop.cpp:153-172, 324-329).
 * The per-light support check the reference makes at each shading point
 * (validate_sampler_support) is not repeated on the device. lights == NULL returns to the
 * scene's CDF selection; bf200_scene_set_light_powers also replaces the tree. A refit keeps the
 * tree as given: set it again with the moved lights' bounds. The adjoint refuses a scene that
 * selects by a tree (INVALID_STATE). */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_scene_set_light_tree(bf200_scene* scene,
                                                                         const bf200_light_tree_input_v1* lights,
                                                                         uint32_t light_count) BF200_NOEXCEPT;
/* bf200_light_tree_select with positions, samples and results in device memory: the tree is built
 * on the host and traversed on the device, one query per thread. Logarithms and exponentials are
 * the double-precision values rounded to float, within about an ulp of the C library's, so a
 * probability may differ from bf200_light_tree_select's in its last bits. Synchronises before
 * returning. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_light_tree_select_device(
    const bf200_light_tree_input_v1* lights, uint32_t light_count, const float* device_positions,
    const float* device_samples, uint64_t query_count, uint32_t* device_light_indices,
    float* device_probabilities) BF200_NOEXCEPT;
/* The tree's probability of selecting light_indices[q] at positions[q] (probability(context, i),
 * LightSampler.cpp:1151-1225); -1 where the reference refuses the query. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_light_tree_probability(const bf200_light_tree_input_v1* lights,
                                                                           uint32_t light_count,
                                                                           const float* positions,
                                                                           const uint32_t* light_indices,
                                                                           uint64_t query_count,
                                                                           float* probabilities) BF200_NOEXCEPT;

/* Triangle-mesh import for callers that hold meshes as OBJ or ASCII PLY files
 * (engine::load_obj_triangle_mesh / load_ply_triangle_mesh, TriangleMeshImport.hpp:9-17): the
 * same files are accepted and refused, and an accepted file gives the same aligned arrays (one
 * vertex per distinct OBJ v/vt/vn corner, in order of first use). The path must be absolute and end
 * in ".obj" or ".ply". On failure `message` (when given) receives the reason. The mesh is host
 * memory owned by the library until bf200_mesh_destroy; its arrays fill one geometry of a
 * bf200_scene_desc_v1. Host code only: no GPU is needed. */
typedef struct bf200_mesh bf200_mesh;

typedef struct bf200_mesh_view_v1 {
    uint32_t struct_size;
    uint32_t vertex_count;
    uint32_t triangle_count;
    uint32_t reserved;
    const float* positions;           /* 3 per vertex */
    const float* normals;             /* 3 per vertex, unit length */
    const float* texture_coordinates; /* 2 per vertex */
    const uint32_t* triangles;        /* 3 per triangle */
} bf200_mesh_view_v1;

BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_mesh_load(const char* absolute_path, bf200_mesh** mesh,
                                                              char* message, uint64_t message_capacity)
    BF200_NOEXCEPT;
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_mesh_view(const bf200_mesh* mesh, bf200_mesh_view_v1* view)
    BF200_NOEXCEPT;
BF200_EXTERN_C BF200_EXPORT void bf200_mesh_destroy(bf200_mesh* mesh) BF200_NOEXCEPT;

/* Closest-hit query for a batch of world rays (trace_cuda_closest_hits, ClosestHit.hpp:21-28).
 * Per ray writes t, barycentrics b0..b2, instance index and primitive index (0xffffffff on a
 * miss). Host pointers. */
typedef struct bf200_hit_v1 {
    float t;
    float barycentrics[3];
    uint32_t instance_index;
    uint32_t primitive_index;
    uint32_t status;
    uint32_t reserved;
} bf200_hit_v1;
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_closest_hits(bf200_context* context,
                                                                  const bf200_scene* scene,
                                                                  const bf200_ray_v1* rays,
                                                                  uint64_t ray_count,
                                                                  bf200_hit_v1* hits)
    BF200_NOEXCEPT;
/* Any-hit query (trace_cuda_occlusions, Occlusion.hpp:19-26): 1 if occluded, else 0. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_occlusions(bf200_context* context,
                                                                const bf200_scene* scene,
                                                                const bf200_ray_v1* rays,
                                                                uint64_t ray_count,
                                                                uint32_t* occluded) BF200_NOEXCEPT;

/* Environment-map light (EnvironmentLights.hpp:468-1075, EnvironmentMapLightT<float>): a
 * packet-bound, piecewise-constant latitude-longitude map, importance-sampled by texel (mean packet
 * radiance times the texel's exact solid angle). Local +Y is north, u = 0 is the +X seam and u
 * grows toward +Z; `environment_to_world` (a unit quaternion x, y, z, w) rotates local directions
 * into world space. bf200_environment_map_create replaces EnvironmentMapLightT::create
 * (EnvironmentLights.hpp:470-733): the sampling tables are built on the host exactly as there and
 * uploaded to the context's device. The batch calls replace sample_li (:750-822), pdf_li
 * (:824-843), le (:845-851) and power (:853-885); like the reference they require the packet the
 * map was created with (`nanometers`, compared exactly), and report each query's failure in its
 * own status (0: the reference returns a value) -- see bf200_environment_status. Host pointers.
 * On the device, sines, cosines and the arctangent are the double-precision values rounded once
 * to float; the reference calls the C library's float functions, which differ by an ulp on a
 * small share of angles. */
typedef struct bf200_environment_map bf200_environment_map;
typedef struct bf200_environment_map_desc_v1 {
    uint32_t struct_size;
    uint32_t width;
    uint32_t height;
    uint32_t reserved;
    const float* texels;             /* width * height records of 4 lanes, row-major, row 0 at +Y */
    float nanometers[4];             /* the wavelength packet the map is bound to */
    float environment_to_world[4];   /* unit quaternion x, y, z, w */
} bf200_environment_map_desc_v1;

/* Per-query status of the batch calls. */
typedef enum bf200_environment_status {
    BF200_ENVIRONMENT_OK = 0,
    BF200_ENVIRONMENT_INVALID_SAMPLE = 1,     /* canonical sample outside [0, 1)^2 */
    BF200_ENVIRONMENT_INVALID_DIRECTION = 2,  /* pdf: not a finite unit vector; le: not representable */
    BF200_ENVIRONMENT_ESCAPED = 3,            /* a lookup escaped its angular partition or CDF */
    BF200_ENVIRONMENT_UNSTABLE = 4,           /* the rotation cannot keep the selected texel */
    BF200_ENVIRONMENT_NOT_REPRESENTABLE = 5   /* an interior sample or its direction is not representable */
} bf200_environment_status;

/* One sample_li: `valid` 0 with status OK is the reference's empty optional (a black map). The
 * sample is infinite: solid-angle pdf, no distance. */
typedef struct bf200_environment_sample_v1 {
    float direction[3];  /* world direction to the light */
    float radiance[4];   /* incident radiance, packet lanes */
    float pdf;           /* solid-angle density */
    uint32_t status;
    uint32_t valid;
} bf200_environment_sample_v1;

BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_environment_map_create(
    bf200_context* context, const bf200_environment_map_desc_v1* desc, bf200_environment_map** map) BF200_NOEXCEPT;
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_environment_map_destroy(bf200_environment_map* map) BF200_NOEXCEPT;
/* canonical: 2 floats (u, v) per query; u picks the column within the row that v picks. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_environment_map_sample(
    bf200_context* context, const bf200_environment_map* map, const float nanometers[4], const float* canonical,
    uint64_t count, bf200_environment_sample_v1* samples) BF200_NOEXCEPT;
/* directions: 3 floats per query (unit vectors toward the light). */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_environment_map_pdf(
    bf200_context* context, const bf200_environment_map* map, const float nanometers[4], const float* directions,
    uint64_t count, float* pdf, uint32_t* status) BF200_NOEXCEPT;
/* directions: 3 floats per query (escaped-ray directions, any length); radiance: 4 per query. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_environment_map_le(
    bf200_context* context, const bf200_environment_map* map, const float nanometers[4], const float* directions,
    uint64_t count, float* radiance, uint32_t* status) BF200_NOEXCEPT;
/* Power over the bounding sphere of the scene bounds [lo, hi] (host arithmetic). */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_environment_map_power(
    bf200_context* context, const bf200_environment_map* map, const float nanometers[4], const float bounds_min[3],
    const float bounds_max[3], float power[4]) BF200_NOEXCEPT;

/* The render interface table returned by get_interface(BF200_RENDER_INTERFACE_ID, 1, 0). */
typedef struct bf200_render_api_v1 {
    uint32_t struct_size;
    uint32_t abi_major;
    uint32_t abi_minor;
    uint32_t reserved;
    blackframe_status (*context_create)(int32_t, uint64_t, bf200_context**) BF200_NOEXCEPT;
    blackframe_status (*context_destroy)(bf200_context*) BF200_NOEXCEPT;
    const char* (*context_last_error)(const bf200_context*) BF200_NOEXCEPT;
    blackframe_status (*scene_create)(bf200_context*, const bf200_scene_desc_v1*,
                                      bf200_scene**) BF200_NOEXCEPT;
    blackframe_status (*scene_destroy)(bf200_scene*) BF200_NOEXCEPT;
    blackframe_status (*trace_paths)(bf200_context*, const bf200_scene*,
                                     const bf200_path_input_v1*, uint64_t,
                                     const bf200_transport_options_v1*, bf200_path_result_v1*,
                                     bf200_report_v1*) BF200_NOEXCEPT;
    blackframe_status (*render_film)(bf200_context*, const bf200_scene*, const bf200_camera_v1*,
                                     const bf200_sensor_v1*, const bf200_film_request_v1*,
                                     const bf200_transport_options_v1*, bf200_film_v1*,
                                     bf200_report_v1*) BF200_NOEXCEPT;
    blackframe_status (*closest_hits)(bf200_context*, const bf200_scene*, const bf200_ray_v1*,
                                      uint64_t, bf200_hit_v1*) BF200_NOEXCEPT;
    blackframe_status (*occlusions)(bf200_context*, const bf200_scene*, const bf200_ray_v1*,
                                    uint64_t, uint32_t*) BF200_NOEXCEPT;
    /* abi_minor 1: the entry points a reference-side adapter needs for the SoA blob and for the
     * cones and initial states of CudaWavefrontPathInput */
    blackframe_status (*scene_create_from_soa)(bf200_context*, const void*, uint64_t, bf200_scene**, char*,
                                               uint64_t) BF200_NOEXCEPT;
    blackframe_status (*trace_paths_with_cones)(bf200_context*, const bf200_scene*, const bf200_path_input_v1*,
                                                const bf200_path_state_v1*, const bf200_ray_cone_v1*, uint64_t,
                                                const bf200_transport_options_v1*, bf200_path_result_v1*,
                                                bf200_ray_cone_v1*, bf200_report_v1*) BF200_NOEXCEPT;
    uint64_t reserved_slots[2];
} bf200_render_api_v1;

/* Derives a pinhole camera the way PinholeCamera::create does (PinholeCamera.hpp:60-99): the
 * orientation frame is OrthonormalFrame::from_normal_and_tangent(normal, tangent_seed)
 * (LocalFrame.hpp:82-89), half_height = tan(vertical_fov / 2), half_width = half_height * W/H. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_camera_create(
    const float origin[3], const float normal[3], const float tangent_seed[3], uint32_t width,
    uint32_t height, float vertical_fov_radians, float time, uint32_t jitter_mode,
    bf200_camera_v1* out_camera) BF200_NOEXCEPT;

/* Stable compaction of one-byte route keys on the device: the wavefront's route queues, which
 * replace the reference's stable appends (blackframe_cuda_launch_wavefront_queue_compaction,
 * WavefrontQueueCompaction.hpp: the slots of one route appended in increasing slot order). Slots
 * whose key is r < routes go to queue[offsets[r] .. offsets[r + 1]) in increasing slot order;
 * other keys (the wavefront's 0xff: no route) are left out. routes: 1..4. Device pointers:
 * keys[count], queue[count], offsets[routes + 1]. Runs on the context's stream and returns when
 * it is done. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_compact_routes_device(
    bf200_context* context, const uint8_t* keys, uint32_t count, uint32_t routes, uint32_t* queue,
    uint32_t* offsets) BF200_NOEXCEPT;

/* Primary rays of (pixel, sample) records through a camera, generated on the context's device by
 * the same code that starts film paths: PinholeCamera::generate_primary_ray with the camera's
 * pixel jitter drawn from the record's sample stream (PinholeCamera.hpp:144-283, PixelJitter.hpp:
 * 47-64). sampler: BF200_SAMPLER_* of the stream. status: 0, or the lane failure code of a ray the
 * reference would refuse. Host pointers. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_camera_rays(
    bf200_context* context, const bf200_camera_v1* camera, const bf200_sample_index_v1* samples,
    uint64_t count, uint32_t sampler, bf200_ray_v1* rays, uint32_t* status) BF200_NOEXCEPT;

/* Sobol coordinate of a sample index in one of the 21,201 Joe-Kuo D6 dimensions, as a 64-bit
 * fixed-point fraction (sobol_sample_bits, SobolSampling.hpp:16-19). Dimensions from 21201 up
 * return BLACKFRAME_STATUS_OUT_OF_RANGE. Host computation. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_sobol_bits(uint64_t sample_index, uint64_t sobol_dimension,
                                                               uint64_t* out_bits) BF200_NOEXCEPT;
/* Owen-scrambled Sobol coordinate of (pixel, sample index, seed) in one Sobol dimension
 * (owen_scrambled_sobol_bits, OwenScrambling.hpp:11-13). Host computation. */
BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_owen_sobol_bits(const bf200_sample_index_v1* index,
                                                                    uint64_t sobol_dimension,
                                                                    uint64_t* out_bits) BF200_NOEXCEPT;

/* BLAS build of the scenes a context creates. BF200_BUILD_HOST_SAH (the default): binned SAH on
 * the host, collapsed to BVH4, like the reference's CudaSceneBvh::build. BF200_BUILD_DEVICE_LBVH:
 * triangle geometries of at least 4,096 triangles are built on the GPU as a linear BVH (Morton
 * order, Karras' hierarchy, leaves of at most four triangles) in a fraction of the time, at some
 * cost in traversal speed; smaller geometries, spheres and the TLAS stay on the host, and a device
 * tree too deep for the traversal stack is rebuilt on the host. Hits are identical either way.
 * Scenes already created keep their build. */
#define BF200_BUILD_HOST_SAH 0u
#define BF200_BUILD_DEVICE_LBVH 1u

BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_context_set_build_mode(bf200_context* context,
                                                                          uint32_t mode) BF200_NOEXCEPT;

/* Build statistics of a scene: its sizes and the host wall time of each phase of
 * bf200_scene_create (BLAS builds, BVH2-to-BVH4 collapse, the instance level with its TLAS and
 * mesh lights, then the uploads and the world-normal kernel). The caller sets struct_size. */
typedef struct bf200_scene_stats_v1 {
    uint32_t struct_size;
    uint32_t blas_depth;              /* deepest BLAS, in BVH4 levels */
    uint32_t device_built_geometries; /* BLASes built on the device (BF200_BUILD_DEVICE_LBVH) */
    uint32_t reserved;
    uint64_t node_count;              /* BVH4 nodes of every BLAS and the TLAS */
    uint64_t leaf_triangle_count;     /* leaf records (triangles and spheres) */
    double blas_build_ms;
    double collapse_ms;
    double instance_ms;
    double upload_ms;
    double total_ms;
} bf200_scene_stats_v1;

BF200_EXTERN_C BF200_EXPORT blackframe_status bf200_scene_stats(const bf200_scene* scene,
                                                               bf200_scene_stats_v1* out) BF200_NOEXCEPT;

/* ---- Native scene JSON (engine::SceneDescriptionJson.hpp, schema "blackframe.scene" v1) ----
 * bf200_scene_json_parse replaces deserialize_scene_description_json
 * (SceneDescriptionJson.hpp:48-50; SceneDescriptionJsonReader.cpp:2430-2457) and
 * bf200_scene_json_write replaces serialize_scene_description_json (:45-47). Both return the
 * reference's core::StatusCode numbering (BF200_SCENE_JSON_*), so a caller sees the same accept or
 * refuse decision and code for the same bytes. A parsed document is the validated
 * SceneDescription (SceneDescription::create's checks included). Host-image textures and
 * normal/bump maps are refused with BF200_SCENE_JSON_UNAVAILABLE: this backend has no image
 * textures. bf200_scene_json_frame turns the active film, camera and render options into the
 * arguments of bf200_scene_create and bf200_render_film. Host computation only. */
typedef struct bf200_scene_json bf200_scene_json;

/* SceneDescriptionJsonLimits (SceneDescriptionJson.hpp:18-33). Every field must be non-zero and
 * at most MaximumSceneDescriptionJsonLimits; a null pointer means the default limits. */
typedef struct bf200_scene_json_limits_v1 {
    uint64_t maximum_encoded_bytes;
    uint64_t maximum_total_values;
    uint64_t maximum_total_string_bytes;
    uint64_t maximum_mesh_vertices;
    uint64_t maximum_mesh_triangles;
    uint64_t maximum_image_scalar_values;
    uint64_t maximum_decoded_bytes;
    uint32_t maximum_nesting_depth;
    uint32_t maximum_records_per_registry;
} bf200_scene_json_limits_v1;

/* core::StatusCode (Status.hpp:10-20). */
#define BF200_SCENE_JSON_OK 0u
#define BF200_SCENE_JSON_INVALID_ARGUMENT 1u
#define BF200_SCENE_JSON_UNAVAILABLE 2u
#define BF200_SCENE_JSON_NOT_FOUND 3u
#define BF200_SCENE_JSON_INCOMPATIBLE 4u
#define BF200_SCENE_JSON_RESOURCE_EXHAUSTED 5u
#define BF200_SCENE_JSON_INTERNAL_ERROR 8u

/* Parses and validates `size` bytes. On success *out_document owns the description; on failure it
 * is null and `message` (when given) holds the reason. */
BF200_EXTERN_C BF200_EXPORT uint32_t bf200_scene_json_parse(const char* bytes, uint64_t size,
                                                            const bf200_scene_json_limits_v1* limits,
                                                            bf200_scene_json** out_document, char* message,
                                                            uint64_t message_capacity) BF200_NOEXCEPT;
BF200_EXTERN_C BF200_EXPORT void bf200_scene_json_destroy(bf200_scene_json* document) BF200_NOEXCEPT;

/* The canonical encoding of a document (the reference writer's bytes for the same description).
 * *out_size receives its length; the bytes are written when out is not null and capacity holds
 * them (BF200_SCENE_JSON_RESOURCE_EXHAUSTED otherwise, with *out_size still set). */
BF200_EXTERN_C BF200_EXPORT uint32_t bf200_scene_json_write(const bf200_scene_json* document,
                                                            const bf200_scene_json_limits_v1* limits, char* out,
                                                            uint64_t capacity, uint64_t* out_size, char* message,
                                                            uint64_t message_capacity) BF200_NOEXCEPT;

/* The active selection of a document, ready to render. `scene` is the committed frame scene
 * (registries in identifier order, instance transforms resolved through the hierarchy as
 * FrameScene::create resolves them, punctual lights in light-registry order, the environment
 * light's packet and radiance); its arrays belong to the document and live until it is destroyed.
 * `camera` is the active pinhole camera over the active film with the render options' pixel
 * jitter; `options` carries the MIS heuristic, depth limits and Russian roulette. The remaining
 * fields echo the film and render options. A render of the document is bf200_scene_create(scene)
 * then bf200_render_film(camera, request {samples_per_pixel, seed, precision}, options) over the
 * full extent; the crop selects the pixels the reference's film covers. */
typedef struct bf200_scene_json_frame_v1 {
    uint32_t struct_size;
    uint32_t film_id;
    uint32_t camera_id;
    uint32_t render_options_id;
    uint32_t width;
    uint32_t height;
    uint32_t crop[4];                 /* minimum x, minimum y, maximum x, maximum y (half-open) */
    uint32_t precision;               /* film accumulation: 0 float32, 1 float64 */
    uint32_t samples_per_pixel;
    uint32_t maximum_path_depth;
    uint32_t tile_edge_length;
    uint32_t light_sampling_strategy; /* 0 uniform, 1 power weighted, 2 spatial tree */
    uint32_t reserved;
    uint64_t seed;
    bf200_camera_v1 camera;
    bf200_transport_options_v1 options;
    bf200_scene_desc_v1 scene;
} bf200_scene_json_frame_v1;

/* Fills *out for the document's active selection. Returns BF200_SCENE_JSON_UNAVAILABLE with a
 * message for a document this backend cannot render: no instances, or no spectral environment
 * light (the packet of a render). */
BF200_EXTERN_C BF200_EXPORT uint32_t bf200_scene_json_frame(const bf200_scene_json* document,
                                                            bf200_scene_json_frame_v1* out, char* message,
                                                            uint64_t message_capacity) BF200_NOEXCEPT;

/* Library version and build description (sm_100a arch string). */
BF200_EXTERN_C BF200_EXPORT const char* bf200_build_info(void) BF200_NOEXCEPT;

#endif /* BF200_H */
