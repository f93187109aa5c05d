"""The BVH-stress workload (985,090 triangles: three displaced subdivision-7 icospheres instanced
40 times, a 2,048-triangle mesh light, a constant environment): closest hits bit-exact and
per-path radiance against the oracle on a sample of the 1920 x 1080 frame's paths."""
import numpy as np
import pytest

from bf200 import abi, runtime, scenes
from helpers import arrays, bit_equal, check_paths
from oracle.bindings import Oracle

pytestmark = pytest.mark.gpu
NAME = "bvh_stress_1080p"


@pytest.fixture(scope="module")
def setup():
    builder, options, (width, height, spp) = scenes.build_workload(NAME)
    oracle = Oracle(device_trig=True)
    handle = oracle.scene(builder)
    with runtime.Context(0, path_capacity=1 << 16) as ctx:
        scene = ctx.create_scene(builder)
        yield builder, options, (width, height, spp), oracle, handle, ctx, scene
        scene.close()
    oracle.destroy(handle)


def test_bvh_stress_closest_hits_bit_exact(setup):
    builder, _, _, oracle, handle, ctx, scene = setup
    rng = np.random.default_rng(21)
    n = 300
    origins = rng.uniform(-14.0, 14.0, (n, 3)).astype(np.float32)
    directions = rng.normal(size=(n, 3)).astype(np.float32)
    directions /= np.linalg.norm(directions, axis=1, keepdims=True)
    rays = (abi.Ray * n)()
    for k in range(n):
        for a in range(3):
            rays[k].origin[a], rays[k].direction[a] = float(origins[k, a]), float(directions[k, a])
        rays[k].t_min, rays[k].t_max, rays[k].time, rays[k].mask = 0.0, float("inf"), 0.5, 0xFFFFFFFF
    expected = oracle.closest_hits(handle, rays)
    got = ctx.closest_hits(scene, rays)
    e_ids = np.array([(h.instance_index, h.primitive_index) for h in expected], np.uint32)
    g_ids = np.array([(h.instance_index, h.primitive_index) for h in got], np.uint32)
    assert (np.array([h.status for h in got]) == 0).all()
    assert (e_ids == g_ids).all(), f"{(e_ids != g_ids).any(axis=1).sum()} hit-ID mismatches"
    assert (e_ids[:, 0] != 0xFFFFFFFF).sum() > n // 5  # the sample really hits geometry
    e_t = np.array([[h.t] + list(h.barycentrics) for h in expected], np.float32)
    g_t = np.array([[h.t] + list(h.barycentrics) for h in got], np.float32)
    assert bit_equal(e_t, g_t).all()


def test_bvh_stress_paths_match_oracle(setup):
    builder, options, (width, height, spp), oracle, handle, ctx, scene = setup
    origin, normal, tangent, vfov = scenes.workload_camera(NAME)
    cam = runtime.camera_create(origin, normal, tangent, width, height, vfov, scenes.PATH_TIME)
    rng = np.random.default_rng(8)
    n = 48
    samples = (abi.SampleIndex * n)()
    for k in range(n):
        samples[k].pixel_x, samples[k].pixel_y = int(rng.integers(width)), int(rng.integers(height))
        samples[k].sample_index = int(rng.integers(spp))
    rays = oracle.camera_rays(cam, samples)
    inputs = (abi.PathInput * n)()
    for k in range(n):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    expected, failures = oracle.trace(handle, inputs, options)
    assert failures == 0
    got, report = ctx.trace_paths(scene, inputs, options)
    assert report.failed_lanes == 0
    check_paths(arrays(got), arrays(expected), NAME)
