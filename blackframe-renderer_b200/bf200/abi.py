"""ctypes mirrors of the records in include/bf200.h.

These are the same byte layouts the C ABI declares; `check_layouts()` asserts the sizes the
header's static assertions expect so a drift between the two is caught on the CPU.
"""
import ctypes as C

u32, u64, f32, f64 = C.c_uint32, C.c_uint64, C.c_float, C.c_double

BLACKFRAME_STATUS = {
    0: "SUCCESS", 1: "INVALID_ARGUMENT", 2: "UNSUPPORTED_ABI", 3: "INTERFACE_NOT_FOUND",
    4: "INVALID_STATE", 5: "OUT_OF_RANGE", 6: "EXTENSION_FAILURE",
}

CLOSURE_LAMBERTIAN = 1
CLOSURE_ROUGH_DIFFUSE = 2
CLOSURE_ROUGH_CONDUCTOR = 3
CLOSURE_ROUGH_DIELECTRIC = 4
CLOSURE_SPECULAR_REFLECTION = 5
CLOSURE_SPECULAR_TRANSMISSION = 6

LOBE_DIFFUSE, LOBE_GLOSSY, LOBE_SPECULAR = 0x01, 0x02, 0x04
LOBE_REFLECTION, LOBE_TRANSMISSION, LOBE_VOLUME = 0x08, 0x10, 0x20

TERMINATIONS = ["escaped_environment", "depth_limit", "outside_bsdf_support",
                "zero_throughput", "russian_roulette"]


class InterfaceId(C.Structure):
    _fields_ = [("high", u64), ("low", u64)]


class Utf8View(C.Structure):
    _fields_ = [("data", C.c_char_p), ("size", u32), ("reserved", u32)]


class ExtensionQuery(C.Structure):
    _fields_ = [("struct_size", u32), ("abi_major", u32), ("abi_minor", u32), ("reserved", u32)]


GetInterfaceFn = C.CFUNCTYPE(u32, C.c_void_p, InterfaceId, u32, u32, C.c_void_p, u32)
ShutdownFn = C.CFUNCTYPE(None, C.c_void_p)


class ExtensionApi(C.Structure):
    _fields_ = [("struct_size", u32), ("abi_major", u32), ("abi_minor", u32), ("reserved", u32),
                ("extension_context", C.c_void_p), ("get_interface", GetInterfaceFn),
                ("shutdown", ShutdownFn)]


class XpuDeviceDescriptor(C.Structure):
    _fields_ = [("struct_size", u32), ("kind", u32), ("identifier_high", u64),
                ("identifier_low", u64), ("name", Utf8View), ("vendor", Utf8View),
                ("reserved", u64 * 4)]


GetDeviceCountFn = C.CFUNCTYPE(u32, C.c_void_p, C.POINTER(u32))
GetDeviceDescriptorFn = C.CFUNCTYPE(u32, C.c_void_p, u32, C.POINTER(XpuDeviceDescriptor))


class XpuBackendApi(C.Structure):
    _fields_ = [("struct_size", u32), ("abi_major", u32), ("abi_minor", u32), ("reserved", u32),
                ("backend_context", C.c_void_p), ("backend_name", Utf8View),
                ("get_device_count", GetDeviceCountFn),
                ("get_device_descriptor", GetDeviceDescriptorFn),
                ("reserved_slots", u64 * 4)]


class Closure(C.Structure):
    _fields_ = [("kind", u32), ("lobes", u32), ("weight", f32 * 4), ("parameters", f32 * 10)]


class Material(C.Structure):
    _fields_ = [("material_id", u32), ("closure_offset", u32), ("closure_count", u32),
                ("frame_mode", u32), ("tangent_rotation_radians", f32),
                ("component_probabilities", f32 * 8), ("emitted_radiance", f32 * 4),
                ("reserved", u32 * 3)]


GEOMETRY_TRIANGLES = 0
GEOMETRY_SPHERE = 1


class Geometry(C.Structure):
    _fields_ = [("geometry_id", u32), ("vertex_offset", u32), ("vertex_count", u32),
                ("triangle_offset", u32), ("triangle_count", u32), ("kind", u32), ("radius", C.c_float),
                ("reserved", u32)]


class Instance(C.Structure):
    _fields_ = [("instance_id", u32), ("object_id", u32), ("geometry_index", u32),
                ("material_index", u32), ("visibility_mask", u32), ("reserved", u32 * 3),
                ("object_to_world", f32 * 16), ("world_to_object", f32 * 16)]


class PunctualLight(C.Structure):
    _fields_ = [("kind", u32), ("reserved", u32), ("position", f32 * 3), ("position_error", f32 * 3),
                ("direction", f32 * 3), ("inner_half_angle", f32), ("outer_half_angle", f32), ("spectrum", f32 * 4)]


PUNCTUAL_POINT, PUNCTUAL_DIRECTIONAL, PUNCTUAL_SPOT = 1, 2, 3


class SceneDesc(C.Structure):
    _fields_ = [("struct_size", u32), ("geometry_count", u32), ("vertex_count", u32),
                ("triangle_count", u32), ("material_count", u32), ("closure_count", u32),
                ("instance_count", u32), ("punctual_light_count", u32),
                ("geometries", C.POINTER(Geometry)), ("positions", C.POINTER(f32)),
                ("normals", C.POINTER(f32)), ("texture_coordinates", C.POINTER(f32)),
                ("triangles", C.POINTER(u32)), ("materials", C.POINTER(Material)),
                ("closures", C.POINTER(Closure)), ("instances", C.POINTER(Instance)),
                ("wavelength_nanometers", f32 * 4), ("wavelength_pdf", f32 * 4),
                ("environment_radiance", f32 * 4), ("reserved", u32 * 4),
                ("punctual_lights", C.POINTER(PunctualLight))]


class Ray(C.Structure):
    _fields_ = [("origin", f32 * 3), ("direction", f32 * 3), ("t_min", f32), ("t_max", f32),
                ("time", f32), ("mask", u32), ("medium", u32), ("reserved", u32)]


class SampleIndex(C.Structure):
    _fields_ = [("pixel_x", u32), ("pixel_y", u32), ("sample_index", u64), ("seed", u64)]


class PathInput(C.Structure):
    _fields_ = [("primary_ray", Ray), ("sample", SampleIndex), ("reserved", u64)]


class PathResult(C.Structure):
    _fields_ = [("beta", f32 * 4), ("radiance", f32 * 4), ("depth", u32),
                ("depth_counters", u32 * 5), ("eta_scale", f32), ("delta_flags", u32),
                ("termination", u32), ("blocked_depth_limits", u32), ("lane_status", u32),
                ("segments", u32), ("terminal_ray", Ray)]


class TransportOptions(C.Structure):
    _fields_ = [("struct_size", u32), ("mis_heuristic", u32), ("depth_limits", u32 * 5),
                ("roulette_enabled", u32), ("roulette_first_eligible_depth", u32),
                ("roulette_minimum_survival", f32), ("roulette_maximum_survival", f32),
                ("instrumentation", u32), ("sampler", u32), ("reserved", u32 * 3)]


class Camera(C.Structure):
    _fields_ = [("origin", f32 * 3), ("tangent", f32 * 3), ("bitangent", f32 * 3),
                ("normal", f32 * 3), ("half_width", f32), ("half_height", f32), ("t_min", f32),
                ("t_max", f32), ("time", f32), ("mask", u32), ("width", u32), ("height", u32),
                ("jitter_mode", u32), ("reserved", u32)]


class Sensor(C.Structure):
    _fields_ = [("response_xyz", (f32 * 3) * 4), ("wavelength_pdf", f32 * 4),
                ("normalization", f32), ("reserved", u32 * 3)]


class FilmRequest(C.Structure):
    _fields_ = [("struct_size", u32), ("samples_per_pixel", u32), ("first_sample", u64),
                ("seed", u64), ("precision", u32), ("reserved", u32 * 3)]


class Film(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("precision", u32), ("reserved", u32),
                ("sums", C.c_void_p), ("sample_counts", C.POINTER(u64))]


class FilmJob(C.Structure):
    _fields_ = [("struct_size", u32), ("reserved", u32), ("scene", C.c_void_p),
                ("camera", C.POINTER(Camera)), ("sensor", C.POINTER(Sensor)),
                ("request", C.POINTER(FilmRequest)), ("options", C.c_void_p), ("film", C.POINTER(Film)),
                ("report", C.c_void_p)]


class MeshView(C.Structure):
    _fields_ = [("struct_size", u32), ("vertex_count", u32), ("triangle_count", u32), ("reserved", u32),
                ("positions", C.POINTER(C.c_float)), ("normals", C.POINTER(C.c_float)),
                ("texture_coordinates", C.POINTER(C.c_float)), ("triangles", C.POINTER(u32))]


class MaterialGradient(C.Structure):
    _fields_ = [("weight", C.c_double * 4), ("roughness", C.c_double * 2), ("reserved", C.c_double * 2)]


class Adjoint(C.Structure):
    _fields_ = [("struct_size", u32), ("reserved", u32), ("target", C.c_void_p), ("gradients", C.c_void_p),
                ("emission_gradient", C.c_void_p), ("loss", C.c_double)]


class Report(C.Structure):
    _fields_ = [("struct_size", u32), ("registered_light_count", u32), ("path_count", u64),
                ("extension_segments", u64), ("shadow_segments", u64),
                ("closure_samples", u64), ("light_samples", u64), ("terminated_paths", u64),
                ("failed_lanes", u64), ("first_failure_status", u32),
                ("first_failure_path", u32), ("kernel_launches", u64),
                ("gpu_milliseconds", f64), ("intersect_milliseconds", f64), ("shade_milliseconds", f64),
                ("occlude_milliseconds", f64), ("film_milliseconds", f64), ("iterations", u64),
                ("regenerate_milliseconds", f64), ("miss_segments", u64), ("continuation_segments", u64)]


class Hit(C.Structure):
    _fields_ = [("t", f32), ("barycentrics", f32 * 3), ("instance_index", u32),
                ("primitive_index", u32), ("status", u32), ("reserved", u32)]


class RayCone(C.Structure):
    """bf200_ray_cone_v1: radius at the ray origin and radial slope."""
    _fields_ = [("width", C.c_float), ("spread", C.c_float)]


class PathState(C.Structure):
    """bf200_path_state_v1: a depth-zero initial path state."""
    _fields_ = [("beta", C.c_float * 4), ("radiance", C.c_float * 4), ("eta_scale", C.c_float),
                ("reserved", C.c_uint32 * 3)]


class LightTreeInput(C.Structure):
    """bf200_light_tree_input_v1: a light's world bounds and four-lane spectral power."""
    _fields_ = [("bounds_min", C.c_float * 3), ("bounds_max", C.c_float * 3), ("spectral_power", C.c_float * 4)]


EXPECTED_SIZES = {
    RayCone: 8, PathState: 48, LightTreeInput: 40,
    Closure: 64, Material: 80, Geometry: 32, Instance: 160, Ray: 48, SampleIndex: 24,
    PathInput: 80, PathResult: 128, TransportOptions: 64, Camera: 88, Sensor: 80,
    FilmRequest: 40, FilmJob: 64, MeshView: 48, MaterialGradient: 64, Adjoint: 40, Report: 152, Hit: 32, ExtensionApi: 40, XpuDeviceDescriptor: 88,
}


def check_layouts():
    for record, size in EXPECTED_SIZES.items():
        actual = C.sizeof(record)
        if actual != size:
            raise AssertionError(f"{record.__name__}: {actual} bytes, header expects {size}")


def default_options(mis="balance", max_depth=8, roulette=True, first_eligible=3,
                    minimum_survival=0.05, maximum_survival=0.95):
    options = TransportOptions()
    options.struct_size = C.sizeof(TransportOptions)
    options.mis_heuristic = 1 if mis == "power" else 0
    for lane in range(4):
        options.depth_limits[lane] = max_depth
    options.depth_limits[4] = 0
    options.roulette_enabled = 1 if roulette else 0
    options.roulette_first_eligible_depth = first_eligible if roulette else 0
    options.roulette_minimum_survival = minimum_survival if roulette else 0.0
    options.roulette_maximum_survival = maximum_survival if roulette else 0.0
    return options


# Native scene JSON (bf200_scene_json_*): core::StatusCode numbering of the codec's results.
SCENE_JSON_CODES = {0: "success", 1: "invalid_argument", 2: "unavailable", 3: "not_found", 4: "incompatible",
                    5: "resource_exhausted", 6: "protocol_error", 7: "platform_error", 8: "internal_error"}


class SceneJsonLimits(C.Structure):
    _fields_ = [("maximum_encoded_bytes", u64), ("maximum_total_values", u64),
                ("maximum_total_string_bytes", u64), ("maximum_mesh_vertices", u64),
                ("maximum_mesh_triangles", u64), ("maximum_image_scalar_values", u64),
                ("maximum_decoded_bytes", u64), ("maximum_nesting_depth", u32),
                ("maximum_records_per_registry", u32)]


class SceneJsonFrame(C.Structure):
    _fields_ = [("struct_size", u32), ("film_id", u32), ("camera_id", u32), ("render_options_id", u32),
                ("width", u32), ("height", u32), ("crop", u32 * 4), ("precision", u32),
                ("samples_per_pixel", u32), ("maximum_path_depth", u32), ("tile_edge_length", u32),
                ("light_sampling_strategy", u32), ("reserved", u32), ("seed", u64), ("camera", Camera),
                ("options", TransportOptions), ("scene", SceneDesc)]


class SceneStats(C.Structure):
    _fields_ = [("struct_size", u32), ("blas_depth", u32), ("device_built_geometries", u32), ("reserved", u32),
                ("node_count", u64), ("leaf_triangle_count", u64), ("blas_build_ms", f64), ("collapse_ms", f64),
                ("instance_ms", f64), ("upload_ms", f64), ("total_ms", f64)]


BUILD_HOST_SAH, BUILD_DEVICE_LBVH = 0, 1
