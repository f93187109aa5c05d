"""Python binding of the bf200 C ABI (include/bf200.h) over ctypes.

This mirrors the reference's call shape for the wavefront path:
  CudaSceneSoA::upload + CudaSceneBvh::build -> Context.create_scene
  trace_cuda_wavefront_transport             -> Context.trace_paths
  caller-side film accumulation              -> Context.render_film
The library is the in-tree bf200/libbf200.so; there is no fallback implementation — if it is
missing or a call fails the error is raised.
"""
import ctypes as C
import os

import numpy as np

from . import abi

_LIB = None
LIBRARY_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libbf200.so")

EXPORTED_SYMBOLS = [
    "blackframe_query_extension", "bf200_context_create", "bf200_context_destroy",
    "bf200_context_last_error", "bf200_scene_create", "bf200_scene_destroy", "bf200_trace_paths",
    "bf200_trace_paths_device", "bf200_render_film", "bf200_render_film_device",
    "bf200_closest_hits", "bf200_occlusions", "bf200_build_info", "bf200_camera_create",
    "bf200_trace_paths_device_noalloc", "bf200_sobol_bits", "bf200_owen_sobol_bits",
    "bf200_render_films_device",
    "bf200_render_adjoint_device",
    "bf200_render_backward_device",
    "bf200_scene_refit",
    "bf200_scene_create_from_soa",
    "bf200_scene_set_light_powers",
    "bf200_light_power_cdf",
    "bf200_mesh_load",
    "bf200_mesh_view",
    "bf200_mesh_destroy",
    "bf200_trace_paths_with_cones",
    "bf200_trace_paths_with_cones_device",
    "bf200_light_tree_select",
    "bf200_light_tree_probability",
    "bf200_light_tree_select_device",
    "bf200_scene_set_light_tree",
    "bf200_environment_map_create",
    "bf200_environment_map_destroy",
    "bf200_environment_map_sample",
    "bf200_environment_map_pdf",
    "bf200_environment_map_le",
    "bf200_environment_map_power",
    "bf200_camera_rays",
    "bf200_compact_routes_device",
    "bf200_scene_json_parse",
    "bf200_scene_json_destroy",
    "bf200_scene_json_write",
    "bf200_scene_json_frame",
    "bf200_scene_stats",
    "bf200_context_set_build_mode",
    "bf200_context_batch_lanes",
]


class Bf200Error(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{abi.BLACKFRAME_STATUS.get(status, status)}: {message}")
        self.status = status


def library():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIBRARY_PATH):
        raise Bf200Error(6, f"{LIBRARY_PATH} is not built (run __graft_entry__.build())")
    lib = C.CDLL(LIBRARY_PATH)
    vp = C.c_void_p
    lib.bf200_build_info.restype = C.c_char_p
    lib.bf200_context_create.argtypes = [C.c_int32, C.c_uint64, C.POINTER(vp)]
    lib.bf200_context_create.restype = C.c_uint32
    lib.bf200_context_destroy.argtypes = [vp]
    lib.bf200_context_destroy.restype = C.c_uint32
    lib.bf200_context_last_error.argtypes = [vp]
    lib.bf200_context_last_error.restype = C.c_char_p
    lib.bf200_scene_create.argtypes = [vp, C.POINTER(abi.SceneDesc), C.POINTER(vp)]
    lib.bf200_scene_create.restype = C.c_uint32
    lib.bf200_scene_destroy.argtypes = [vp]
    lib.bf200_scene_destroy.restype = C.c_uint32
    for name in ("bf200_trace_paths", "bf200_trace_paths_device"):
        f = getattr(lib, name)
        f.argtypes = [vp, vp, vp, C.c_uint64, C.POINTER(abi.TransportOptions), vp, C.POINTER(abi.Report)]
        f.restype = C.c_uint32
    lib.bf200_trace_paths_device_noalloc.argtypes = [vp, vp, vp, C.c_uint64, C.POINTER(abi.TransportOptions), vp,
                                                     C.c_uint32, C.POINTER(abi.Report)]
    lib.bf200_trace_paths_device_noalloc.restype = C.c_uint32
    for f in (lib.bf200_trace_paths_with_cones, lib.bf200_trace_paths_with_cones_device):
        f.argtypes = [vp, vp, vp, vp, vp, C.c_uint64, C.POINTER(abi.TransportOptions), vp, vp, C.POINTER(abi.Report)]
        f.restype = C.c_uint32
    for name in ("bf200_render_film", "bf200_render_film_device"):
        f = getattr(lib, name)
        f.argtypes = [vp, vp, C.POINTER(abi.Camera), C.POINTER(abi.Sensor), C.POINTER(abi.FilmRequest),
                      C.POINTER(abi.TransportOptions), C.POINTER(abi.Film), C.POINTER(abi.Report)]
        f.restype = C.c_uint32
    lib.bf200_closest_hits.argtypes = [vp, vp, vp, C.c_uint64, vp]
    lib.bf200_closest_hits.restype = C.c_uint32
    lib.bf200_occlusions.argtypes = [vp, vp, vp, C.c_uint64, vp]
    lib.bf200_occlusions.restype = C.c_uint32
    lib.bf200_camera_create.argtypes = [C.POINTER(C.c_float)] * 3 + [C.c_uint32, C.c_uint32, C.c_float,
                                                                      C.c_float, C.c_uint32, C.POINTER(abi.Camera)]
    lib.bf200_camera_create.restype = C.c_uint32
    lib.bf200_render_films_device.argtypes = [vp, C.POINTER(abi.FilmJob), C.c_uint32, C.c_uint32]
    lib.bf200_render_films_device.restype = C.c_uint32
    lib.bf200_render_adjoint_device.argtypes = [vp, vp, C.POINTER(abi.Camera), C.POINTER(abi.Sensor),
                                                C.POINTER(abi.FilmRequest), C.POINTER(abi.TransportOptions),
                                                C.POINTER(abi.Film), C.POINTER(abi.Adjoint), C.POINTER(abi.Report)]
    lib.bf200_render_adjoint_device.restype = C.c_uint32
    lib.bf200_render_backward_device.argtypes = [vp, vp, C.POINTER(abi.Camera), C.POINTER(abi.Sensor),
                                                 C.POINTER(abi.FilmRequest), C.POINTER(abi.TransportOptions),
                                                 C.POINTER(abi.Film), vp, vp, vp, C.POINTER(abi.Report)]
    lib.bf200_render_backward_device.restype = C.c_uint32
    lib.bf200_scene_set_light_powers.argtypes = [vp, vp, C.c_uint32]
    lib.bf200_scene_set_light_powers.restype = C.c_uint32
    lib.bf200_light_power_cdf.argtypes = [vp, C.c_uint32, vp]
    lib.bf200_light_power_cdf.restype = C.c_uint32
    lib.bf200_scene_create_from_soa.argtypes = [vp, vp, C.c_uint64, C.POINTER(vp), C.c_char_p, C.c_uint64]
    lib.bf200_scene_create_from_soa.restype = C.c_uint32
    lib.bf200_scene_refit.argtypes = [vp, C.POINTER(abi.SceneDesc)]
    lib.bf200_scene_refit.restype = C.c_uint32
    lib.bf200_mesh_load.argtypes = [C.c_char_p, C.POINTER(vp), C.c_char_p, C.c_uint64]
    lib.bf200_mesh_load.restype = C.c_uint32
    lib.bf200_mesh_view.argtypes = [vp, C.POINTER(abi.MeshView)]
    lib.bf200_mesh_view.restype = C.c_uint32
    lib.bf200_mesh_destroy.argtypes = [vp]
    lib.bf200_mesh_destroy.restype = None
    lib.bf200_sobol_bits.argtypes = [C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]
    lib.bf200_sobol_bits.restype = C.c_uint32
    lib.bf200_owen_sobol_bits.argtypes = [C.POINTER(abi.SampleIndex), C.c_uint64, C.POINTER(C.c_uint64)]
    lib.bf200_owen_sobol_bits.restype = C.c_uint32
    lib.blackframe_query_extension.argtypes = [C.POINTER(abi.ExtensionQuery), C.POINTER(abi.ExtensionApi)]
    lib.blackframe_query_extension.restype = C.c_uint32
    _LIB = lib
    return lib


def query_extension():
    """blackframe_query_extension as a Blackframe host calls it (XpuBackend.cpp:57-100)."""
    lib = library()
    query = abi.ExtensionQuery(C.sizeof(abi.ExtensionQuery), 1, 0, 0)
    api = abi.ExtensionApi()
    api.struct_size = C.sizeof(abi.ExtensionApi)
    status = lib.blackframe_query_extension(C.byref(query), C.byref(api))
    return status, api


class Scene:
    def __init__(self, context, handle, builder):
        self.context = context
        self.handle = handle
        self.builder = builder

    def set_light_powers(self, powers):
        """bf200_scene_set_light_powers: power-weighted selection from 4-lane spectral powers per
        light (None: uniform again)."""
        if powers is None:
            lights = sum(1 for inst in self.builder.instances if any(v != 0 for v in self.builder.materials[inst[1]][1]))
            status = library().bf200_scene_set_light_powers(self.handle, None, lights)
        else:
            powers = np.ascontiguousarray(powers, np.float32).reshape(-1, 4)
            status = library().bf200_scene_set_light_powers(self.handle, powers.ctypes.data_as(C.c_void_p),
                                                            len(powers))
        self.context._check(status, "scene_set_light_powers")

    def refit(self, builder, desc=None):
        """bf200_scene_refit with `builder`'s description (or `desc`, already made from it): only
        instance transforms may differ."""
        desc = builder.desc() if desc is None else desc
        self.context._check(library().bf200_scene_refit(self.handle, C.byref(desc)), "scene_refit")
        self.builder = builder

    def set_light_tree(self, lights):
        """bf200_scene_set_light_tree: select lights by the spatial tree of `lights` (an array of
        abi.LightTreeInput in registry order), or by the scene's CDF again with None."""
        f = library().bf200_scene_set_light_tree
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
        f.restype = C.c_uint32
        status = f(self.handle, C.cast(lights, C.c_void_p) if lights is not None else None,
                   len(lights) if lights is not None else 0)
        if status != 0:
            raise Bf200Error(status, "set_light_tree")

    def stats(self):
        """bf200_scene_stats: sizes and the host wall time of each scene-creation phase (abi.SceneStats)."""
        out = abi.SceneStats()
        out.struct_size = C.sizeof(out)
        f = library().bf200_scene_stats
        f.argtypes = [C.c_void_p, C.POINTER(abi.SceneStats)]
        f.restype = C.c_uint32
        if f(self.handle, C.byref(out)) != 0:
            raise Bf200Error(1, "scene_stats")
        return out

    def close(self):
        if self.handle:
            library().bf200_scene_destroy(self.handle)
            self.handle = None


class Context:
    def __init__(self, device=0, path_capacity=0):
        lib = library()
        handle = C.c_void_p()
        status = lib.bf200_context_create(device, path_capacity, C.byref(handle))
        if status != 0:
            raise Bf200Error(status, f"context creation on device {device} failed")
        self.handle = handle

    def _check(self, status, what):
        if status != 0:
            message = library().bf200_context_last_error(self.handle)
            raise Bf200Error(status, f"{what}: {message.decode() if message else ''}")

    def close(self):
        if self.handle:
            library().bf200_context_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def batch_lanes(self):
        """bf200_context_batch_lanes: the lane count of the last render_films_device call."""
        out = C.c_uint32()
        f = library().bf200_context_batch_lanes
        f.argtypes = [C.c_void_p, C.POINTER(C.c_uint32)]
        f.restype = C.c_uint32
        self._check(f(self.handle, C.byref(out)), "context_batch_lanes")
        return out.value

    def set_build_mode(self, mode):
        """bf200_context_set_build_mode: abi.BUILD_HOST_SAH (default) or abi.BUILD_DEVICE_LBVH for the
        scenes created from now on."""
        f = library().bf200_context_set_build_mode
        f.argtypes = [C.c_void_p, C.c_uint32]
        f.restype = C.c_uint32
        self._check(f(self.handle, mode), "context_set_build_mode")

    def create_scene(self, builder, desc=None):
        """bf200_scene_create from `builder`'s description (or `desc`, already made from it)."""
        desc = builder.desc() if desc is None else desc
        handle = C.c_void_p()
        self._check(library().bf200_scene_create(self.handle, C.byref(desc), C.byref(handle)), "scene")
        return Scene(self, handle, builder)

    def create_scene_from_soa(self, blob, builder=None):
        """bf200_scene_create_from_soa from a scene SoA v4 blob (bytes)."""
        handle = C.c_void_p()
        message = C.create_string_buffer(512)
        data = C.create_string_buffer(bytes(blob), len(blob))
        status = library().bf200_scene_create_from_soa(self.handle, data, len(blob), C.byref(handle), message,
                                                        len(message))
        if status != 0:
            raise Bf200Error(status, message.value.decode(errors="replace"))
        return Scene(self, handle, builder)

    def trace_paths(self, scene, inputs, options):
        n = len(inputs)
        results = (abi.PathResult * n)()
        report = abi.Report()
        report.struct_size = C.sizeof(abi.Report)
        self._check(library().bf200_trace_paths(self.handle, scene.handle, C.cast(inputs, C.c_void_p), n,
                                                C.byref(options), C.cast(results, C.c_void_p),
                                                C.byref(report)), "trace_paths")
        return results, report

    def trace_paths_with_cones(self, scene, inputs, cones, options, states=None):
        """bf200_trace_paths_with_cones: cones is float32 [n, 2] of primary (width, spread); states
        (optional) an array of abi.PathState; returns (results, terminal cones float32 [n, 2],
        report)."""
        import numpy as np
        n = len(inputs)
        cones = np.ascontiguousarray(cones, np.float32).reshape(n, 2)
        terminal = np.zeros((n, 2), np.float32)
        results = (abi.PathResult * n)()
        report = abi.Report()
        report.struct_size = C.sizeof(abi.Report)
        self._check(library().bf200_trace_paths_with_cones(
            self.handle, scene.handle, C.cast(inputs, C.c_void_p),
            C.cast(states, C.c_void_p) if states is not None else None, cones.ctypes.data_as(C.c_void_p), n,
            C.byref(options), C.cast(results, C.c_void_p), terminal.ctypes.data_as(C.c_void_p), C.byref(report)),
            "trace_paths_with_cones")
        return results, terminal, report

    def trace_paths_with_cones_device(self, scene, device_inputs, device_cones, path_count, options,
                                      device_results, device_terminal_cones, device_states=None):
        """bf200_trace_paths_with_cones_device: every array is a device pointer (int); device_states
        may be None (every path starts from the initial state)."""
        report = abi.Report()
        report.struct_size = C.sizeof(abi.Report)
        self._check(library().bf200_trace_paths_with_cones_device(
            self.handle, scene.handle, device_inputs, device_states, device_cones, path_count, C.byref(options),
            device_results, device_terminal_cones, C.byref(report)), "trace_paths_with_cones_device")
        return report

    def trace_paths_device(self, scene, device_inputs, path_count, options, device_results):
        """bf200_trace_paths_device: inputs and results are device pointers (ints)."""
        report = abi.Report()
        report.struct_size = C.sizeof(abi.Report)
        self._check(library().bf200_trace_paths_device(self.handle, scene.handle, device_inputs, path_count,
                                                       C.byref(options), device_results, C.byref(report)),
                    "trace_paths_device")
        return report

    def trace_paths_device_noalloc(self, scene, device_inputs, path_count, options, device_results,
                                   path_capacity=0):
        """bf200_trace_paths_device_noalloc: the allocation-free variant over the library's static
        scratch array (path_capacity slots, 0 = the maximum)."""
        report = abi.Report()
        report.struct_size = C.sizeof(abi.Report)
        self._check(library().bf200_trace_paths_device_noalloc(self.handle, scene.handle, device_inputs, path_count,
                                                               C.byref(options), device_results, path_capacity,
                                                               C.byref(report)),
                    "trace_paths_device_noalloc")
        return report

    def render_films_device(self, jobs, lanes=0):
        """bf200_render_films_device. `jobs`: (scene, camera, sensor, options, samples_per_pixel,
        seed, first_sample, precision, sums_ptr, counts_ptr) tuples with device film pointers.
        Returns one report per job."""
        n = len(jobs)
        records = (abi.FilmJob * n)()
        keep = []
        reports = [abi.Report() for _ in range(n)]
        for k, (scene, camera, sensor, options, spp, seed, first, precision, sums, counts) in enumerate(jobs):
            request = abi.FilmRequest(C.sizeof(abi.FilmRequest), spp, first, seed, precision)
            film = abi.Film(camera.width, camera.height, precision, 0, C.c_void_p(sums),
                            C.cast(C.c_void_p(counts), C.POINTER(abi.u64)))
            keep += [request, film, camera, sensor, options]
            r = records[k]
            r.struct_size = C.sizeof(abi.FilmJob)
            r.scene = scene.handle
            r.camera = C.pointer(camera)
            r.sensor = C.pointer(sensor)
            r.request = C.pointer(request)
            r.options = C.cast(C.pointer(options), C.c_void_p)
            r.film = C.pointer(film)
            reports[k].struct_size = C.sizeof(abi.Report)
            r.report = C.cast(C.pointer(reports[k]), C.c_void_p)
        self._check(library().bf200_render_films_device(self.handle, records, n, lanes), "render_films_device")
        return reports

    def render_film_device(self, scene, camera, sensor, options, samples_per_pixel, seed, first_sample, precision,
                           sums, counts):
        """bf200_render_film_device with device film pointers; returns the report."""
        request = abi.FilmRequest(C.sizeof(abi.FilmRequest), samples_per_pixel, first_sample, seed, precision)
        film = abi.Film(camera.width, camera.height, precision, 0, C.c_void_p(sums),
                        C.cast(C.c_void_p(counts), C.POINTER(abi.u64)))
        report = abi.Report()
        report.struct_size = C.sizeof(abi.Report)
        self._check(library().bf200_render_film_device(self.handle, scene.handle, C.byref(camera), C.byref(sensor),
                                                       C.byref(request), C.byref(options), C.byref(film),
                                                       C.byref(report)), "render_film_device")
        return report

    def render_adjoint_device(self, scene, camera, sensor, options, samples_per_pixel, seed, first_sample, precision,
                              sums, counts, target, gradients, emission_gradient):
        """bf200_render_adjoint_device: renders the device film (cleared first) and writes the loss
        gradients (`gradients`: one 8-double record per material, `emission_gradient`: one double;
        device pointers, as is `target`, H x W x 3 floats). Returns (loss, report)."""
        request = abi.FilmRequest(C.sizeof(abi.FilmRequest), samples_per_pixel, first_sample, seed, precision)
        film = abi.Film(camera.width, camera.height, precision, 0, C.c_void_p(sums),
                        C.cast(C.c_void_p(counts), C.POINTER(abi.u64)))
        adjoint = abi.Adjoint(C.sizeof(abi.Adjoint), 0, C.c_void_p(target), C.c_void_p(gradients),
                              C.c_void_p(emission_gradient), 0.0)
        report = abi.Report()
        report.struct_size = C.sizeof(abi.Report)
        self._check(library().bf200_render_adjoint_device(self.handle, scene.handle, C.byref(camera),
                                                          C.byref(sensor), C.byref(request), C.byref(options),
                                                          C.byref(film), C.byref(adjoint), C.byref(report)),
                    "render_adjoint_device")
        return adjoint.loss, report

    def render_backward_device(self, scene, camera, sensor, options, samples_per_pixel, seed, first_sample,
                               precision, sums, counts, image_adjoint, gradients, emission_gradient):
        """bf200_render_backward_device: gradients for dLoss/d(image) = `image_adjoint` (device,
        H x W x 3 floats) of the film that render_film_device wrote to (sums, counts) with the same
        arguments. Returns the report of the re-trace."""
        request = abi.FilmRequest(C.sizeof(abi.FilmRequest), samples_per_pixel, first_sample, seed, precision)
        film = abi.Film(camera.width, camera.height, precision, 0, C.c_void_p(sums),
                        C.cast(C.c_void_p(counts), C.POINTER(abi.u64)))
        report = abi.Report()
        report.struct_size = C.sizeof(abi.Report)
        self._check(library().bf200_render_backward_device(self.handle, scene.handle, C.byref(camera),
                                                           C.byref(sensor), C.byref(request), C.byref(options),
                                                           C.byref(film), C.c_void_p(image_adjoint),
                                                           C.c_void_p(gradients), C.c_void_p(emission_gradient),
                                                           C.byref(report)), "render_backward_device")
        return report

    def render_film(self, scene, camera, sensor, options, samples_per_pixel, seed=0, first_sample=0,
                    precision=0, film=None):
        """Adds (pixel, sample) paths for samples [first_sample, first_sample + spp) to a film.

        Returns (sums, counts, report): sums is float32 [H, W, 4] (r, g, b, weight) or float64
        [H, W, 8] (sums, compensations) for precision 1.
        """
        w, h = camera.width, camera.height
        if film is None:
            sums = np.zeros((h, w, 4 if precision == 0 else 8), np.float32 if precision == 0 else np.float64)
            counts = np.zeros((h, w), np.uint64)
        else:
            sums, counts = film
        f = abi.Film(w, h, precision, 0, sums.ctypes.data_as(C.c_void_p),
                     counts.ctypes.data_as(C.POINTER(abi.u64)))
        request = abi.FilmRequest(C.sizeof(abi.FilmRequest), samples_per_pixel, first_sample, seed, precision)
        report = abi.Report()
        report.struct_size = C.sizeof(abi.Report)
        self._check(library().bf200_render_film(self.handle, scene.handle, C.byref(camera), C.byref(sensor),
                                                C.byref(request), C.byref(options), C.byref(f),
                                                C.byref(report)), "render_film")
        return sums, counts, report

    def compact_routes_device(self, keys_ptr, count, routes, queue_ptr, offsets_ptr):
        """bf200_compact_routes_device on device buffers (uint8 keys, uint32 queue and offsets)."""
        lib = library()
        lib.bf200_compact_routes_device.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                                    C.c_void_p]
        self._check(lib.bf200_compact_routes_device(self.handle, keys_ptr, count, routes, queue_ptr, offsets_ptr),
                    "compact_routes_device")

    def camera_rays(self, camera, samples, sampler=0):
        """Primary rays of abi.SampleIndex records through `camera` (abi.Camera), generated on the
        device; returns (abi.Ray array, numpy uint32 statuses)."""
        n = len(samples)
        rays = (abi.Ray * n)()
        status = np.zeros(n, np.uint32)
        lib = library()
        lib.bf200_camera_rays.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p,
                                          C.c_void_p]
        self._check(lib.bf200_camera_rays(self.handle, C.byref(camera), C.cast(samples, C.c_void_p), n, sampler,
                                          C.cast(rays, C.c_void_p), status.ctypes.data_as(C.c_void_p)),
                    "camera_rays")
        return rays, status

    def closest_hits(self, scene, rays):
        n = len(rays)
        hits = (abi.Hit * n)()
        self._check(library().bf200_closest_hits(self.handle, scene.handle, C.cast(rays, C.c_void_p), n,
                                                 C.cast(hits, C.c_void_p)), "closest_hits")
        return hits

    def occlusions(self, scene, rays):
        n = len(rays)
        out = np.zeros(n, np.uint32)
        self._check(library().bf200_occlusions(self.handle, scene.handle, C.cast(rays, C.c_void_p), n,
                                               out.ctypes.data_as(C.c_void_p)), "occlusions")
        return out


def light_power_cdf(powers):
    """bf200_light_power_cdf: the light_count + 1 selection boundaries of 4-lane spectral powers."""
    powers = np.ascontiguousarray(powers, np.float32).reshape(-1, 4)
    out = np.zeros(len(powers) + 1, np.float32)
    status = library().bf200_light_power_cdf(powers.ctypes.data_as(C.c_void_p), len(powers),
                                             out.ctypes.data_as(C.c_void_p))
    if status != 0:
        raise Bf200Error(status, "light power CDF refused")
    return out



def _light_tree_inputs(bounds_min, bounds_max, powers):
    import numpy as np
    bounds_min = np.ascontiguousarray(bounds_min, np.float32).reshape(-1, 3)
    bounds_max = np.ascontiguousarray(bounds_max, np.float32).reshape(-1, 3)
    powers = np.ascontiguousarray(powers, np.float32).reshape(-1, 4)
    lights = (abi.LightTreeInput * len(powers))()
    for k in range(len(powers)):
        lights[k].bounds_min[:] = [float(v) for v in bounds_min[k]]
        lights[k].bounds_max[:] = [float(v) for v in bounds_max[k]]
        lights[k].spectral_power[:] = [float(v) for v in powers[k]]
    return lights


def light_tree_select(bounds_min, bounds_max, powers, positions, samples):
    """bf200_light_tree_select: (selected slots uint32, probabilities float32); a refused query
    gives 0xFFFFFFFF and -1. Raises Bf200Error when the tree itself is refused."""
    import numpy as np
    lights = _light_tree_inputs(bounds_min, bounds_max, powers)
    positions = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    samples = np.ascontiguousarray(samples, np.float32)
    selected = np.zeros(len(samples), np.uint32)
    probabilities = np.zeros(len(samples), np.float32)
    f = library().bf200_light_tree_select
    f.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    f.restype = C.c_uint32
    status = f(C.cast(lights, C.c_void_p), len(lights), positions.ctypes.data_as(C.c_void_p),
               samples.ctypes.data_as(C.c_void_p), len(samples), selected.ctypes.data_as(C.c_void_p),
               probabilities.ctypes.data_as(C.c_void_p))
    if status != 0:
        raise Bf200Error(status, "light tree refused")
    return selected, probabilities


def light_tree_select_device(bounds_min, bounds_max, powers, device_positions, device_samples, query_count,
                             device_light_indices, device_probabilities):
    """bf200_light_tree_select_device: positions, samples and outputs are device pointers (ints)."""
    lights = _light_tree_inputs(bounds_min, bounds_max, powers)
    f = library().bf200_light_tree_select_device
    f.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    f.restype = C.c_uint32
    status = f(C.cast(lights, C.c_void_p), len(lights), device_positions, device_samples, query_count,
               device_light_indices, device_probabilities)
    if status != 0:
        raise Bf200Error(status, "light tree refused")


def light_tree_probability(bounds_min, bounds_max, powers, positions, light_indices):
    """bf200_light_tree_probability: float32 probabilities (-1 where a query is refused)."""
    import numpy as np
    lights = _light_tree_inputs(bounds_min, bounds_max, powers)
    positions = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    light_indices = np.ascontiguousarray(light_indices, np.uint32)
    probabilities = np.zeros(len(light_indices), np.float32)
    f = library().bf200_light_tree_probability
    f.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]
    f.restype = C.c_uint32
    status = f(C.cast(lights, C.c_void_p), len(lights), positions.ctypes.data_as(C.c_void_p),
               light_indices.ctypes.data_as(C.c_void_p), len(light_indices), probabilities.ctypes.data_as(C.c_void_p))
    if status != 0:
        raise Bf200Error(status, "light tree refused")
    return probabilities


def load_mesh(path):
    """bf200_mesh_load: an OBJ or ASCII PLY file as (positions [V, 3], normals [V, 3], texture
    coordinates [V, 2], triangles [T, 3]) numpy arrays; raises Bf200Error when the file is refused."""
    lib = library()
    handle = C.c_void_p()
    message = C.create_string_buffer(512)
    status = lib.bf200_mesh_load(os.fsencode(path), C.byref(handle), message, len(message))
    if status != 0:
        raise Bf200Error(status, message.value.decode(errors="replace"))
    try:
        view = abi.MeshView()
        view.struct_size = C.sizeof(abi.MeshView)
        lib.bf200_mesh_view(handle, C.byref(view))
        nv, nt = view.vertex_count, view.triangle_count
        return (np.ctypeslib.as_array(view.positions, (nv, 3)).copy(),
                np.ctypeslib.as_array(view.normals, (nv, 3)).copy(),
                np.ctypeslib.as_array(view.texture_coordinates, (nv, 2)).copy(),
                np.ctypeslib.as_array(view.triangles, (nt, 3)).copy())
    finally:
        lib.bf200_mesh_destroy(handle)


def camera_create(origin, normal, tangent_seed, width, height, vfov, time=0.5, jitter=1):
    """bf200_camera_create: a pinhole camera derived exactly as PinholeCamera::create does."""
    f3 = lambda a: (C.c_float * 3)(*[float(x) for x in a])
    cam = abi.Camera()
    status = library().bf200_camera_create(f3(origin), f3(normal), f3(tangent_seed), width, height,
                                           vfov, time, jitter, C.byref(cam))
    if status != 0:
        raise Bf200Error(status, "camera creation")
    return cam


def sobol_bits(sample_index, sobol_dimension):
    """bf200_sobol_bits: the 64-bit Sobol coordinate (sobol_sample_bits)."""
    out = C.c_uint64()
    status = library().bf200_sobol_bits(sample_index, sobol_dimension, C.byref(out))
    if status != 0:
        raise Bf200Error(status, f"Sobol dimension {sobol_dimension}")
    return out.value


def owen_sobol_bits(pixel_x, pixel_y, sample_index, seed, sobol_dimension):
    """bf200_owen_sobol_bits: the Owen-scrambled Sobol coordinate (owen_scrambled_sobol_bits)."""
    index = abi.SampleIndex(pixel_x, pixel_y, sample_index, seed)
    out = C.c_uint64()
    status = library().bf200_owen_sobol_bits(C.byref(index), sobol_dimension, C.byref(out))
    if status != 0:
        raise Bf200Error(status, f"Sobol dimension {sobol_dimension}")
    return out.value
