"""ctypes bindings of the CPU checkers (test infrastructure only).

* Oracle: oracle/liboracle.so, this repository's restatement of the reference scalar path tracer
  (oracle/bfo_oracle.cpp).
* Reference: oracle/_ref/libbfref.so, the reference's own sources compiled by oracle/Makefile
  with a thin harness (oracle/ref_harness.cpp). Present only where it was built.

Only tests, __graft_entry__.smoke() and bench.py's CPU arms use these, as checkers; the product
never loads them.
"""
import ctypes as C
import os
import sys

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(ORACLE_DIR)
sys.path.insert(0, os.path.join(REPO, "blackframe-renderer_b200"))

from bf200 import abi  # noqa: E402

ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle.so")
REFERENCE_LIB = os.path.join(ORACLE_DIR, "_ref", "libbfref.so")


class CheckerError(RuntimeError):
    pass


class _Checker:
    prefix = ""

    def __init__(self, path):
        if not os.path.exists(path):
            raise CheckerError(f"{path} is not built")
        self.lib = C.CDLL(path)
        p = self.prefix
        getattr(self.lib, p + "_last_error").restype = C.c_char_p
        f = getattr(self.lib, p + "_scene_create")
        f.argtypes = [C.POINTER(abi.SceneDesc), C.POINTER(C.c_void_p)]
        f.restype = C.c_int
        getattr(self.lib, p + "_scene_destroy").argtypes = [C.c_void_p]
        f = getattr(self.lib, p + "_trace_paths")
        f.argtypes = [C.c_void_p, C.POINTER(abi.PathInput), C.c_uint64, C.POINTER(abi.TransportOptions),
                      C.POINTER(abi.PathResult), C.c_int]
        f.restype = C.c_int64

    def last_error(self):
        return getattr(self.lib, self.prefix + "_last_error")().decode()

    def scene(self, builder, desc=None):
        desc = builder.desc() if desc is None else desc
        handle = C.c_void_p()
        rc = getattr(self.lib, self.prefix + "_scene_create")(C.byref(desc), C.byref(handle))
        if rc != 0:
            raise CheckerError(f"scene creation failed ({rc}): {self.last_error()}")
        return handle

    def destroy(self, handle):
        getattr(self.lib, self.prefix + "_scene_destroy")(handle)

    def sphere_intersect(self, spheres, rays):
        """Ray k against sphere k (centre xyz, radius): float32 [n, 8] of status (0 miss, 1 hit,
        2 not representable), t, outward normal xyz, position xyz."""
        import numpy as np
        spheres = np.ascontiguousarray(spheres, np.float32).reshape(-1, 4)
        out = np.zeros((len(rays), 8), np.float32)
        f = getattr(self.lib, self.prefix + "_sphere_intersect")
        f.argtypes = [C.c_void_p, C.POINTER(abi.Ray), C.c_uint64, C.c_void_p]
        f.restype = C.c_int
        f(spheres.ctypes.data_as(C.c_void_p), rays, len(rays), out.ctypes.data_as(C.c_void_p))
        return out

    def set_light_powers(self, handle, powers):
        """Power-weighted light selection for the scene from 4-lane spectral powers per light."""
        import numpy as np
        powers = np.ascontiguousarray(powers, np.float32).reshape(-1, 4)
        f = getattr(self.lib, self.prefix + "_scene_set_light_powers")
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
        f.restype = C.c_int
        if f(handle, powers.ctypes.data_as(C.c_void_p), len(powers)) != 0:
            raise CheckerError(self.last_error())

    def cone_scatter(self, cones, kinds, parameters, events, wo, wi):
        """propagate_ray_cone_scattering per case: float32 [n, 2] of (width, spread), NaN where it
        fails, and the failure count."""
        import numpy as np
        arrays = [np.ascontiguousarray(cones, np.float32), np.ascontiguousarray(kinds, np.uint32),
                  np.ascontiguousarray(parameters, np.float32), np.ascontiguousarray(events, np.uint32),
                  np.ascontiguousarray(wo, np.float32), np.ascontiguousarray(wi, np.float32)]
        n = len(arrays[1])
        out = np.zeros((n, 2), np.float32)
        f = getattr(self.lib, self.prefix + "_cone_scatter")
        f.argtypes = [C.c_void_p] * 6 + [C.c_uint64, C.c_void_p]
        f.restype = C.c_int64
        failures = f(*[a.ctypes.data_as(C.c_void_p) for a in arrays], n, out.ctypes.data_as(C.c_void_p))
        return out, failures

    def set_light_tree(self, handle, lights):
        """Selection (and MIS) by the spatial light tree of `lights`, an array of
        abi.LightTreeInput in registry order."""
        f = getattr(self.lib, self.prefix + "_scene_set_light_tree")
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
        f.restype = C.c_int
        if f(handle, C.cast(lights, C.c_void_p), len(lights)) != 0:
            raise CheckerError(self.last_error())

    def _before_trace(self):
        pass

    def trace(self, handle, inputs, options, threads=None):
        self._before_trace()
        n = len(inputs)
        results = (abi.PathResult * n)()
        threads = threads or os.cpu_count() or 1
        failures = getattr(self.lib, self.prefix + "_trace_paths")(handle, inputs, n, C.byref(options), results, threads)
        if failures < 0:
            raise CheckerError(self.last_error())
        return results, failures


class Oracle(_Checker):
    """The restatement. device_trig=True rounds the sine and cosine of sampled angles as the device
    does (the float nearest to the double value) instead of as the C library's float functions,
    which the reference calls: the checker of the device path is then exact on every path whose
    other arithmetic is."""
    prefix = "bfo"

    def __init__(self, device_trig=False):
        super().__init__(ORACLE_LIB)
        self.device_trig = bool(device_trig)
        self.lib.bfo_set_device_trig.argtypes = [C.c_int]
        f = self.lib.bfo_film_accumulate
        f.argtypes = [C.c_void_p, C.POINTER(abi.SampleIndex), C.c_uint64, C.POINTER(abi.Sensor), C.c_uint32,
                      C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
        f.restype = C.c_int
        self.lib.bfo_closest_hits.argtypes = [C.c_void_p, C.POINTER(abi.Ray), C.c_uint64, C.POINTER(abi.Hit)]
        self.lib.bfo_scene_world_normal.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(C.c_float)]
        self.lib.bfo_scene_set_prefilter.argtypes = [C.c_void_p, C.c_int]
        self.lib.bfo_camera_rays_sampled.argtypes = [C.POINTER(abi.Camera), C.POINTER(abi.SampleIndex), C.c_uint64,
                                                     C.c_uint32, C.POINTER(abi.Ray)]
        self.lib.bfo_camera_rays_sampled.restype = C.c_int
        self.lib.bfo_sobol_bits.argtypes = [C.c_uint64, C.c_uint64]
        self.lib.bfo_sobol_bits.restype = C.c_uint64
        self.lib.bfo_owen_sobol_bits.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64]
        self.lib.bfo_owen_sobol_bits.restype = C.c_uint64

    def _before_trace(self):
        self.lib.bfo_set_device_trig(1 if self.device_trig else 0)

    def cone_advance(self, cones, directions, parameters):
        """advance_ray_cone_to_hit per case: the advanced widths (NaN where it fails) and the
        failure count."""
        import numpy as np
        cones = np.ascontiguousarray(cones, np.float32)
        directions = np.ascontiguousarray(directions, np.float32)
        parameters = np.ascontiguousarray(parameters, np.float32)
        out = np.zeros(len(parameters), np.float32)
        f = self.lib.bfo_cone_advance
        f.argtypes = [C.c_void_p] * 3 + [C.c_uint64, C.c_void_p]
        f.restype = C.c_int64
        failures = f(cones.ctypes.data_as(C.c_void_p), directions.ctypes.data_as(C.c_void_p),
                     parameters.ctypes.data_as(C.c_void_p), len(parameters), out.ctypes.data_as(C.c_void_p))
        return out, failures

    def trace_cones(self, handle, inputs, cones, options, states=None, threads=None):
        """trace() carrying ray cones and, optionally, depth-zero initial states (an array of
        abi.PathState): (results, terminal cones float32 [n, 2], failures)."""
        import numpy as np
        self._before_trace()
        n = len(inputs)
        cones = np.ascontiguousarray(cones, np.float32).reshape(n, 2)
        results = (abi.PathResult * n)()
        out = np.zeros((n, 2), np.float32)
        f = self.lib.bfo_trace_paths_cones
        f.argtypes = [C.c_void_p, C.POINTER(abi.PathInput), C.c_void_p, C.c_void_p, C.c_uint64,
                      C.POINTER(abi.TransportOptions), C.POINTER(abi.PathResult), C.c_void_p, C.c_int]
        f.restype = C.c_int64
        failures = f(handle, inputs, C.cast(states, C.c_void_p) if states is not None else None,
                     cones.ctypes.data_as(C.c_void_p), n, C.byref(options), results,
                     out.ctypes.data_as(C.c_void_p), threads or os.cpu_count() or 1)
        if failures < 0:
            raise CheckerError(self.last_error())
        return results, out, failures

    def camera_rays(self, camera, samples, sampler=0):
        rays = (abi.Ray * len(samples))()
        if self.lib.bfo_camera_rays_sampled(C.byref(camera), samples, len(samples), sampler, rays) != 0:
            raise CheckerError(self.last_error())
        return rays

    def sobol_bits(self, sample_index, dimension):
        return self.lib.bfo_sobol_bits(sample_index, dimension)

    def owen_sobol_bits(self, px, py, sample_index, seed, dimension):
        return self.lib.bfo_owen_sobol_bits(px, py, sample_index, seed, dimension)

    def closest_hits(self, handle, rays):
        hits = (abi.Hit * len(rays))()
        self.lib.bfo_closest_hits(handle, rays, len(rays), hits)
        return hits

    def weight_gradients(self, handle, inputs, options, path_adjoint, materials):
        """Float64 dLoss/d(closure weight) per material and lane, and dLoss/d(emitter scale), along
        the oracle's paths, from dLoss/dL per path and lane (bfo_weight_gradients)."""
        import numpy as np
        self._before_trace()
        adj = np.ascontiguousarray(path_adjoint, np.float64).reshape(len(inputs), 4)
        grads = np.zeros((materials, 4), np.float64)
        emission = C.c_double()
        f = self.lib.bfo_weight_gradients
        f.argtypes = [C.c_void_p, C.POINTER(abi.PathInput), C.c_uint64, C.POINTER(abi.TransportOptions), C.c_void_p,
                      C.c_void_p, C.POINTER(C.c_double)]
        f.restype = C.c_int64
        failures = f(handle, inputs, len(inputs), C.byref(options), adj.ctypes.data_as(C.c_void_p),
                     grads.ctypes.data_as(C.c_void_p), C.byref(emission))
        return grads, emission.value, failures

    def film(self, radiance, samples, sensor, width, height, precision):
        import numpy as np
        n = len(samples)
        sums = np.zeros((height, width, 4), np.float64)
        counts = np.zeros((height, width), np.uint64)
        rad = np.ascontiguousarray(radiance, np.float32)
        rc = self.lib.bfo_film_accumulate(rad.ctypes.data_as(C.c_void_p), samples, n, C.byref(sensor), width,
                                          height, precision, sums.ctypes.data_as(C.c_void_p),
                                          counts.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise CheckerError("film accumulation failed")
        return sums, counts


class Reference(_Checker):
    prefix = "bfr"

    def power_sampler(self, powers, samples):
        """The reference's power-weighted LightSampler: (probability of every light, selected index
        and probability for every canonical sample), or (None, StatusCode) when it refuses."""
        import numpy as np
        powers = np.ascontiguousarray(powers, np.float32).reshape(-1, 4)
        samples = np.ascontiguousarray(samples, np.float32)
        probabilities = np.zeros(len(powers), np.float32)
        selected = np.zeros(len(samples), np.uint32)
        selected_probability = np.zeros(len(samples), np.float32)
        f = self.lib.bfr_power_sampler
        f.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        f.restype = C.c_int
        code = f(powers.ctypes.data_as(C.c_void_p), len(powers), probabilities.ctypes.data_as(C.c_void_p),
                 samples.ctypes.data_as(C.c_void_p), len(samples), selected.ctypes.data_as(C.c_void_p),
                 selected_probability.ctypes.data_as(C.c_void_p))
        if code != 0:
            return None, code
        return (probabilities, selected, selected_probability), 0

    def trace_states(self, handle, inputs, states, options, threads=None):
        """trace_scene_mis from a depth-zero initial PathState per path (an array of
        abi.PathState): (results, failures)."""
        n = len(inputs)
        results = (abi.PathResult * n)()
        f = self.lib.bfr_trace_paths_states
        f.argtypes = [C.c_void_p, C.POINTER(abi.PathInput), C.c_void_p, C.c_uint64, C.POINTER(abi.TransportOptions),
                      C.POINTER(abi.PathResult), C.c_int]
        f.restype = C.c_int64
        failures = f(handle, inputs, C.cast(states, C.c_void_p), n, C.byref(options), results,
                     threads or os.cpu_count() or 1)
        if failures < 0:
            raise CheckerError(self.last_error())
        return results, failures

    def light_tree(self, bounds_min, bounds_max, powers, positions, samples=None, light_indices=None):
        """The reference's spatial light tree at query points: with samples, (selected slots,
        probabilities) of sample(context, u); with light_indices, (light_indices, probabilities)
        of probability(context, i). Refused queries give 0xFFFFFFFF / -1. Returns (None, code)
        when the tree itself is refused."""
        import numpy as np
        bounds_min = np.ascontiguousarray(bounds_min, np.float32).reshape(-1, 3)
        bounds_max = np.ascontiguousarray(bounds_max, np.float32).reshape(-1, 3)
        powers = np.ascontiguousarray(powers, np.float32).reshape(-1, 4)
        positions = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        n = len(positions)
        mode = 0 if samples is not None else 1
        samples = np.ascontiguousarray(samples if samples is not None else np.zeros(n), np.float32)
        selected = np.ascontiguousarray(light_indices if light_indices is not None else np.zeros(n), np.uint32).copy()
        probabilities = np.zeros(n, np.float32)
        f = self.lib.bfr_light_tree
        f.argtypes = [C.c_void_p] * 3 + [C.c_uint32, C.c_int] + [C.c_void_p] * 2 + [C.c_uint64] + [C.c_void_p] * 2
        f.restype = C.c_int
        code = f(bounds_min.ctypes.data_as(C.c_void_p), bounds_max.ctypes.data_as(C.c_void_p),
                 powers.ctypes.data_as(C.c_void_p), len(powers), mode, positions.ctypes.data_as(C.c_void_p),
                 samples.ctypes.data_as(C.c_void_p), n, selected.ctypes.data_as(C.c_void_p),
                 probabilities.ctypes.data_as(C.c_void_p))
        if code != 0:
            return None, code
        return (selected, probabilities), 0

    def cone_advance(self, cones, distances):
        """renderer::advance_ray_cone(cone, distance) per case: widths (NaN on error), errors."""
        import numpy as np
        cones = np.ascontiguousarray(cones, np.float32)
        distances = np.ascontiguousarray(distances, np.float32)
        out = np.zeros(len(distances), np.float32)
        f = self.lib.bfr_cone_advance
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]
        f.restype = C.c_int64
        failures = f(cones.ctypes.data_as(C.c_void_p), distances.ctypes.data_as(C.c_void_p), len(distances),
                     out.ctypes.data_as(C.c_void_p))
        return out, failures

    def camera_cones(self, origin, normal, tangent, width, height, vfov, time, samples):
        """PinholeCamera::generate_primary_ray_cone for every sample: float32 [n, 2]."""
        import numpy as np
        out = np.zeros((len(samples), 2), np.float32)
        f = self.lib.bfr_camera_cones
        f.argtypes = [C.POINTER(C.c_float)] * 3 + [C.c_uint32, C.c_uint32, C.c_float, C.c_float,
                                                  C.POINTER(abi.SampleIndex), C.c_uint64, C.c_void_p]
        f.restype = C.c_int
        if f(self._f3(origin), self._f3(normal), self._f3(tangent), width, height, vfov, time, samples,
             len(samples), out.ctypes.data_as(C.c_void_p)) != 0:
            raise CheckerError(self.last_error())
        return out

    def load_mesh(self, path):
        """The reference's own OBJ/PLY loader: (positions, normals, uvs, triangles) as numpy arrays,
        or (None, reference status code, message) when it refuses the file."""
        import numpy as np
        f = self.lib.bfr_mesh_load
        f.argtypes = [C.c_char_p, C.POINTER(C.c_int)]
        f.restype = C.c_void_p
        code = C.c_int(0)
        handle = f(path.encode(), C.byref(code))
        if not handle:
            return None, code.value, self.last_error()
        nv, nt = C.c_uint32(), C.c_uint32()
        self.lib.bfr_mesh_counts.argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        self.lib.bfr_mesh_counts(handle, C.byref(nv), C.byref(nt))
        p = np.zeros((nv.value, 3), np.float32)
        n = np.zeros((nv.value, 3), np.float32)
        uv = np.zeros((nv.value, 2), np.float32)
        t = np.zeros((nt.value, 3), np.uint32)
        self.lib.bfr_mesh_copy.argtypes = [C.c_void_p] * 5
        self.lib.bfr_mesh_copy(handle, p.ctypes.data_as(C.c_void_p), n.ctypes.data_as(C.c_void_p),
                               uv.ctypes.data_as(C.c_void_p), t.ctypes.data_as(C.c_void_p))
        self.lib.bfr_mesh_free.argtypes = [C.c_void_p]
        self.lib.bfr_mesh_free(handle)
        return (p, n, uv, t), 0, ""

    def __init__(self):
        super().__init__(REFERENCE_LIB)
        f = self.lib.bfr_camera_rays
        f.argtypes = [C.POINTER(C.c_float)] * 3 + [C.c_uint32, C.c_uint32, C.c_float, C.c_float,
                                                  C.POINTER(abi.SampleIndex), C.c_uint64, C.POINTER(abi.Ray)]
        f.restype = C.c_int
        f = self.lib.bfr_camera
        f.argtypes = [C.POINTER(C.c_float)] * 3 + [C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_float,
                                                  C.c_float, C.c_uint32, C.POINTER(abi.Camera)]
        f.restype = C.c_int
        self.lib.bfr_sensor.argtypes = [C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(abi.Sensor)]
        self.lib.bfr_scene_world_to_object.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(C.c_float)]
        f = self.lib.bfr_film_accumulate
        f.argtypes = [C.c_void_p, C.POINTER(abi.SampleIndex), C.c_uint64, C.POINTER(C.c_float),
                      C.POINTER(C.c_float), C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
        f.restype = C.c_int

    def sobol_bits(self, sample_index, dimension):
        f = self.lib.bfr_sobol_bits
        f.argtypes = [C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]
        f.restype = C.c_int
        out = C.c_uint64()
        if f(sample_index, dimension, C.byref(out)) != 0:
            raise CheckerError(self.last_error())
        return out.value

    def owen_sobol_bits(self, px, py, sample_index, seed, dimension):
        f = self.lib.bfr_owen_sobol_bits
        f.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]
        f.restype = C.c_int
        out = C.c_uint64()
        if f(px, py, sample_index, seed, dimension, C.byref(out)) != 0:
            raise CheckerError(self.last_error())
        return out.value

    @staticmethod
    def _f3(values):
        return (C.c_float * 3)(*[float(v) for v in values])

    def camera_rays(self, origin, normal, tangent, width, height, vfov, time, samples):
        rays = (abi.Ray * len(samples))()
        rc = self.lib.bfr_camera_rays(self._f3(origin), self._f3(normal), self._f3(tangent), width, height, vfov,
                                      time, samples, len(samples), rays)
        if rc != 0:
            raise CheckerError(self.last_error())
        return rays

    def camera(self, origin, normal, tangent, width, height, vfov, time):
        cam = abi.Camera()
        rc = self.lib.bfr_camera(self._f3(origin), self._f3(normal), self._f3(tangent), width, height, vfov, 0.0,
                                 float("inf"), time, 0xFFFFFFFF, C.byref(cam))
        if rc != 0:
            raise CheckerError(self.last_error())
        return cam

    def sensor(self, nanometers, pdfs):
        out = abi.Sensor()
        nm = (C.c_float * 4)(*[float(v) for v in nanometers])
        pdf = (C.c_float * 4)(*[float(v) for v in pdfs])
        self.lib.bfr_sensor(nm, pdf, C.byref(out))
        return out

    def world_to_object(self, handle, index):
        out = (C.c_float * 16)()
        self.lib.bfr_scene_world_to_object(handle, index, out)
        return list(out)

    def film(self, radiance, samples, nanometers, pdfs, width, height, precision):
        import numpy as np
        sums = np.zeros((height, width, 4), np.float64)
        counts = np.zeros((height, width), np.uint64)
        rad = np.ascontiguousarray(radiance, np.float32)
        nm = (C.c_float * 4)(*[float(v) for v in nanometers])
        pdf = (C.c_float * 4)(*[float(v) for v in pdfs])
        rc = self.lib.bfr_film_accumulate(rad.ctypes.data_as(C.c_void_p), samples, len(samples), nm, pdf, width,
                                          height, precision, sums.ctypes.data_as(C.c_void_p),
                                          counts.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise CheckerError(self.last_error())
        return sums, counts


def reference_available():
    return os.path.exists(REFERENCE_LIB)


REFERENCE_CUDA_LIB = os.path.join(ORACLE_DIR, "_ref", "libbfrefcuda.so")


def reference_cuda_available():
    return os.path.exists(REFERENCE_CUDA_LIB)


class ReferenceCuda:
    """oracle/_ref/libbfrefcuda.so: the reference's own CUDA backend (CudaSceneSoA::upload,
    CudaSceneBvh::build, trace_cuda_closest_hits, trace_cuda_wavefront_transport with a reused
    workspace), compiled unchanged for sm_100a by oracle/Makefile. Needs a GPU."""

    def __init__(self):
        if not reference_cuda_available():
            raise CheckerError(f"{REFERENCE_CUDA_LIB} is not built")
        self.lib = C.CDLL(REFERENCE_CUDA_LIB)
        self.lib.bfrc_last_error.restype = C.c_char_p
        self.lib.bfrc_scene_create.argtypes = [C.POINTER(abi.SceneDesc), C.POINTER(C.c_void_p)]
        self.lib.bfrc_scene_create.restype = C.c_int
        self.lib.bfrc_scene_destroy.argtypes = [C.c_void_p]
        self.lib.bfrc_scene_stats.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                              C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        self.lib.bfrc_closest_hits.argtypes = [C.c_void_p, C.POINTER(abi.Ray), C.c_uint64, C.POINTER(abi.Hit)]
        self.lib.bfrc_closest_hits.restype = C.c_int
        self.lib.bfrc_trace.argtypes = [C.c_void_p, C.POINTER(abi.PathInput), C.c_void_p, C.c_uint64,
                                        C.POINTER(abi.TransportOptions), C.c_void_p, C.POINTER(abi.Report),
                                        C.POINTER(C.c_double)]
        self.lib.bfrc_trace.restype = C.c_int

    def last_error(self):
        return self.lib.bfrc_last_error().decode()

    def scene(self, builder, desc=None):
        desc = desc if desc is not None else builder.desc()
        handle = C.c_void_p()
        rc = self.lib.bfrc_scene_create(C.byref(desc), C.byref(handle))
        if rc != 0:
            raise CheckerError(f"reference CUDA scene creation failed ({rc}): {self.last_error()}")
        return handle

    def destroy(self, handle):
        self.lib.bfrc_scene_destroy(handle)

    def stats(self, handle):
        up, build = C.c_double(), C.c_double()
        sb, bb = C.c_uint64(), C.c_uint64()
        self.lib.bfrc_scene_stats(handle, C.byref(up), C.byref(build), C.byref(sb), C.byref(bb))
        return {"upload_ms": up.value, "bvh_build_ms": build.value, "scene_bytes": sb.value, "bvh_bytes": bb.value}

    def closest_hits(self, handle, rays):
        hits = (abi.Hit * len(rays))()
        if self.lib.bfrc_closest_hits(handle, rays, len(rays), hits) != 0:
            raise CheckerError(self.last_error())
        return hits

    def trace(self, handle, inputs, options, cones=None, results=True):
        """One trace_cuda_wavefront_transport call: (results or None, report, host milliseconds)."""
        import numpy as np
        n = len(inputs)
        out = (abi.PathResult * n)() if results else None
        report = abi.Report()
        ms = C.c_double()
        c = np.ascontiguousarray(cones, np.float32).reshape(n, 2) if cones is not None else None
        rc = self.lib.bfrc_trace(handle, inputs, c.ctypes.data_as(C.c_void_p) if c is not None else None, n,
                                 C.byref(options), C.cast(out, C.c_void_p) if out is not None else None,
                                 C.byref(report), C.byref(ms))
        if rc != 0:
            raise CheckerError(self.last_error())
        return out, report, ms.value


class EnvironmentCheck:
    """An environment-map light on the CPU: the oracle's restatement (liboracle.so, prefix "bfo",
    trig rounding chosen by device_trig) or the reference's own EnvironmentMapLightT<float>
    (libbfref.so, prefix "bfref"). Same call shapes as bf200.envmap.EnvironmentMap; creation
    failures raise CheckerError with the code (1 invalid argument, 2 resource exhausted)."""

    def __init__(self, path, prefix, texels, nanometers, quaternion=(0.0, 0.0, 0.0, 1.0), device_trig=False):
        import numpy as np
        if not os.path.exists(path):
            raise CheckerError(f"{path} is not built")
        self.np = np
        self.lib = C.CDLL(path)
        self.prefix = prefix
        self.device_trig = bool(device_trig)
        vp, u64 = C.c_void_p, C.c_uint64
        create = getattr(self.lib, prefix + "_envmap_create")
        create.argtypes = [C.c_uint32, C.c_uint32, vp, vp, vp, C.POINTER(C.c_int), C.c_char_p, C.c_size_t]
        create.restype = vp
        getattr(self.lib, prefix + "_envmap_destroy").argtypes = [vp]
        trig = [C.c_int] if prefix == "bfo" else []
        getattr(self.lib, prefix + "_envmap_sample").argtypes = [vp, vp, u64] + trig + [vp]
        getattr(self.lib, prefix + "_envmap_pdf").argtypes = [vp, vp, u64] + trig + [vp, vp]
        getattr(self.lib, prefix + "_envmap_le").argtypes = [vp, vp, u64] + trig + [vp, vp]
        power = getattr(self.lib, prefix + "_envmap_power")
        power.argtypes = [vp, vp, vp, vp]
        power.restype = C.c_int
        self.texels = np.ascontiguousarray(texels, np.float32)
        height, width, _ = self.texels.shape
        nm = np.ascontiguousarray(nanometers, np.float32).reshape(4)
        q = np.ascontiguousarray(quaternion, np.float32).reshape(4)
        code = C.c_int(0)
        message = C.create_string_buffer(256)
        self.handle = create(width, height, self._ptr(self.texels), self._ptr(nm), self._ptr(q), C.byref(code), message,
                             256)
        if not self.handle:
            self.code = code.value
            raise CheckerError(f"{code.value}: {message.value.decode()}")

    @staticmethod
    def _ptr(a):
        return a.ctypes.data_as(C.c_void_p)

    def _trig(self):
        return [int(self.device_trig)] if self.prefix == "bfo" else []

    def sample(self, canonical):
        from bf200.envmap import SAMPLE_DTYPE
        u = self.np.ascontiguousarray(canonical, self.np.float32).reshape(-1, 2)
        out = self.np.zeros(len(u), SAMPLE_DTYPE)
        getattr(self.lib, self.prefix + "_envmap_sample")(self.handle, self._ptr(u), len(u), *self._trig(),
                                                          self._ptr(out))
        return out

    def pdf(self, directions):
        d = self.np.ascontiguousarray(directions, self.np.float32).reshape(-1, 3)
        pdf, status = self.np.zeros(len(d), self.np.float32), self.np.zeros(len(d), self.np.uint32)
        getattr(self.lib, self.prefix + "_envmap_pdf")(self.handle, self._ptr(d), len(d), *self._trig(), self._ptr(pdf),
                                                       self._ptr(status))
        return pdf, status

    def le(self, directions):
        d = self.np.ascontiguousarray(directions, self.np.float32).reshape(-1, 3)
        radiance = self.np.zeros((len(d), 4), self.np.float32)
        status = self.np.zeros(len(d), self.np.uint32)
        getattr(self.lib, self.prefix + "_envmap_le")(self.handle, self._ptr(d), len(d), *self._trig(),
                                                      self._ptr(radiance), self._ptr(status))
        return radiance, status

    def power(self, lo, hi):
        """(status, power[4]); status 0 when the call returns a value."""
        lo = self.np.ascontiguousarray(lo, self.np.float32).reshape(3)
        hi = self.np.ascontiguousarray(hi, self.np.float32).reshape(3)
        out = self.np.zeros(4, self.np.float32)
        rc = getattr(self.lib, self.prefix + "_envmap_power")(self.handle, self._ptr(lo), self._ptr(hi), self._ptr(out))
        return rc, out

    def close(self):
        if self.handle:
            getattr(self.lib, self.prefix + "_envmap_destroy")(self.handle)
            self.handle = None


def oracle_environment(texels, nanometers, quaternion=(0.0, 0.0, 0.0, 1.0), device_trig=False):
    return EnvironmentCheck(ORACLE_LIB, "bfo", texels, nanometers, quaternion, device_trig)


def reference_environment(texels, nanometers, quaternion=(0.0, 0.0, 0.0, 1.0)):
    return EnvironmentCheck(REFERENCE_LIB, "bfref", texels, nanometers, quaternion)
