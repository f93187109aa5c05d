"""Generates the committed golden fixtures from the reference implementation itself.

Runs only where the reference tree is available to build oracle/_ref/libbfref.so (the reference's
own Core/Renderer/Engine sources + oracle/ref_harness.cpp). For each Cornell workload it stores:
  * the reference pinhole camera (frame and half extents) and the CIE sensor constants of the
    frame's wavelength packet;
  * every instance's committed world_to_object matrix (FrameScene's own inverse);
  * a seeded set of (pixel, sample) path inputs with the reference camera rays, and the
    reference trace_scene_mis results for them;
  * a small film rendered by the reference path (camera rays, trace, CIE XYZ -> linear RGB ->
    Film/ReferenceFilm::add_sample), in float32 and in compensated float64.

Usage: python tests/golden/make_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "blackframe-renderer_b200"))
sys.path.insert(0, REPO)

from bf200 import abi, scenes  # noqa: E402
from oracle.bindings import Reference  # noqa: E402

PLANS = {
    # workload: (path count, film width, film height, film spp)
    "cornell_plain_64": (1024, 64, 64, 2),
    "cornell_spheres_256": (192, 24, 24, 1),
}


def sample_plan(width, height, spp, count, seed):
    rng = np.random.default_rng(seed)
    px = rng.integers(0, width, count)
    py = rng.integers(0, height, count)
    s = rng.integers(0, spp, count)
    return px, py, s


def make_samples(px, py, s, seed=0):
    samples = (abi.SampleIndex * len(px))()
    for k in range(len(px)):
        samples[k].pixel_x, samples[k].pixel_y = int(px[k]), int(py[k])
        samples[k].sample_index, samples[k].seed = int(s[k]), seed
    return samples


def results_arrays(results):
    n = len(results)
    out = {
        "radiance": np.array([list(r.radiance) for r in results], np.float32).reshape(n, 4),
        "beta": np.array([list(r.beta) for r in results], np.float32).reshape(n, 4),
        "depth": np.array([r.depth for r in results], np.uint32),
        "counters": np.array([list(r.depth_counters) for r in results], np.uint32).reshape(n, 5),
        "eta": np.array([r.eta_scale for r in results], np.float32),
        "termination": np.array([r.termination for r in results], np.uint32),
        "blocked": np.array([r.blocked_depth_limits for r in results], np.uint32),
        "lane_status": np.array([r.lane_status for r in results], np.uint32),
        "terminal_origin": np.array([list(r.terminal_ray.origin) for r in results], np.float32).reshape(n, 3),
        "terminal_direction": np.array([list(r.terminal_ray.direction) for r in results], np.float32).reshape(n, 3),
    }
    return out


def camera_array(cam):
    return np.array(list(cam.origin) + list(cam.tangent) + list(cam.bitangent) + list(cam.normal) +
                    [cam.half_width, cam.half_height], np.float32)


def main():
    ref = Reference()
    for name, (count, fw, fh, fspp) in PLANS.items():
        builder, options, (width, height, spp) = scenes.build_workload(name)
        handle = ref.scene(builder)
        origin, normal, tangent = scenes.camera_frame_inputs()
        camera = ref.camera(origin, normal, tangent, width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
        sensor = ref.sensor(builder.nanometers, builder.pdfs)
        px, py, s = sample_plan(width, height, spp, count, seed=7)
        samples = make_samples(px, py, s)
        rays = ref.camera_rays(origin, normal, tangent, width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME,
                               samples)
        inputs = (abi.PathInput * count)()
        for k in range(count):
            inputs[k].primary_ray = rays[k]
            inputs[k].sample = samples[k]
        results, failures = ref.trace(handle, inputs, options)
        print(f"{name}: {count} paths, reference failures {failures}")
        ray_origin = np.array([list(r.origin) for r in rays], np.float32).reshape(count, 3)
        ray_direction = np.array([list(r.direction) for r in rays], np.float32).reshape(count, 3)
        # small film through the reference caller-side loop
        fpx, fpy, fs = np.meshgrid(np.arange(fw), np.arange(fh), np.arange(fspp), indexing="ij")
        order = np.lexsort((fpx.ravel(), fpy.ravel(), fs.ravel()))  # sample-major, then row, column
        fpx, fpy, fs = fpx.ravel()[order], fpy.ravel()[order], fs.ravel()[order]
        film_samples = make_samples(fpx, fpy, fs)
        film_rays = ref.camera_rays(origin, normal, tangent, fw, fh, scenes.CAMERA_VFOV, scenes.PATH_TIME,
                                    film_samples)
        film_inputs = (abi.PathInput * len(fpx))()
        for k in range(len(fpx)):
            film_inputs[k].primary_ray = film_rays[k]
            film_inputs[k].sample = film_samples[k]
        film_results, film_failures = ref.trace(handle, film_inputs, options)
        film_radiance = np.array([list(r.radiance) for r in film_results], np.float32).reshape(-1, 4)
        film32, counts32 = ref.film(film_radiance, film_samples, builder.nanometers, builder.pdfs, fw, fh, 0)
        film64, counts64 = ref.film(film_radiance, film_samples, builder.nanometers, builder.pdfs, fw, fh, 1)
        film_camera = ref.camera(origin, normal, tangent, fw, fh, scenes.CAMERA_VFOV, scenes.PATH_TIME)
        world_to_object = np.array([ref.world_to_object(handle, i) for i in range(len(builder.instances))],
                                   np.float32)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            camera=camera_array(camera), film_camera=camera_array(film_camera),
            sensor_response=np.array([list(r) for r in sensor.response_xyz], np.float32),
            sensor_pdf=np.array(list(sensor.wavelength_pdf), np.float32),
            sensor_normalization=np.float32(sensor.normalization),
            nanometers=np.array(builder.nanometers, np.float32), world_to_object=world_to_object,
            pixel_x=px.astype(np.uint32), pixel_y=py.astype(np.uint32), sample_index=s.astype(np.uint64),
            ray_origin=ray_origin, ray_direction=ray_direction, reference_failures=np.int64(failures),
            film_size=np.array([fw, fh, fspp], np.uint32), film32=film32, counts32=counts32, film64=film64,
            counts64=counts64, film_failures=np.int64(film_failures),
            **results_arrays(results))
        ref.destroy(handle)
        print(f"  film {fw}x{fh}x{fspp}: reference failures {film_failures}")


if __name__ == "__main__":
    main()
