"""The Owen-scrambled Sobol transport sampler (BF200_SAMPLER_OWEN_SOBOL) on the device against the
oracle running the same sampler: per-path radiance on fresh seeds and a full plain frame's film,
with the parity tolerances of the hash-sampler tests."""
import os

import numpy as np
import pytest

from bf200 import abi, runtime, scenes
from helpers import DIVERGED_FRACTION, RELATIVE_TOLERANCE, arrays, check_paths, relative_error, sensor_from_golden
from oracle.bindings import Oracle

pytestmark = pytest.mark.gpu
OWEN = 1


@pytest.fixture(scope="module")
def ctx():
    with runtime.Context(0, path_capacity=1 << 18) as c:
        yield c


def _inputs(oracle, cam, width, height, spp, n, seed):
    rng = np.random.default_rng(seed)
    samples = (abi.SampleIndex * n)()
    for k in range(n):
        samples[k].pixel_x, samples[k].pixel_y = int(rng.integers(width)), int(rng.integers(height))
        samples[k].sample_index, samples[k].seed = int(rng.integers(1 << 20)), 0x243F6A8885A308D3
    rays = oracle.camera_rays(cam, samples, sampler=OWEN)
    inputs = (abi.PathInput * n)()
    for k in range(n):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    return inputs


@pytest.mark.parametrize("name", ["cornell_plain_64", "cornell_spheres_256"])
def test_owen_sobol_paths_match_oracle(ctx, name):
    oracle = Oracle(device_trig=True)
    builder, options, (width, height, spp) = scenes.build_workload(name)
    options.sampler = OWEN
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    inputs = _inputs(oracle, cam, width, height, spp, 2048 if name == "cornell_plain_64" else 512, seed=606)
    handle = oracle.scene(builder)
    expected, failures = oracle.trace(handle, inputs, options)
    oracle.destroy(handle)
    assert failures == 0
    scene = ctx.create_scene(builder)
    got, report = ctx.trace_paths(scene, inputs, options)
    scene.close()
    assert report.failed_lanes == 0
    check_paths(arrays(got), arrays(expected), name + " owen-sobol")


def test_owen_sobol_plain_frame_film_matches_oracle(ctx):
    oracle = Oracle(device_trig=True)
    builder, options, (width, height, spp) = scenes.build_workload("cornell_plain_64")
    options.sampler = OWEN
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cornell_plain_64.npz"))
    sensor = sensor_from_golden(g)
    scene = ctx.create_scene(builder)
    sums, counts, report = ctx.render_film(scene, cam, sensor, options, spp, seed=0)
    hash_options = scenes.build_workload("cornell_plain_64")[1]
    hash_sums, _, _ = ctx.render_film(scene, cam, sensor, hash_options, spp, seed=0)
    scene.close()
    px, py, s = np.meshgrid(np.arange(width), np.arange(height), np.arange(spp), indexing="ij")
    order = np.lexsort((px.ravel(), py.ravel(), s.ravel()))
    px, py, s = px.ravel()[order], py.ravel()[order], s.ravel()[order]
    samples = (abi.SampleIndex * len(px))()
    for k in range(len(px)):
        samples[k].pixel_x, samples[k].pixel_y, samples[k].sample_index = int(px[k]), int(py[k]), int(s[k])
    rays = oracle.camera_rays(cam, samples, sampler=OWEN)
    inputs = (abi.PathInput * len(px))()
    for k in range(len(px)):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    handle = oracle.scene(builder)
    results, failures = oracle.trace(handle, inputs, options)
    oracle.destroy(handle)
    expected, _ = oracle.film(arrays(results)["radiance"], samples, sensor, width, height, 0)
    assert failures == 0 and report.failed_lanes == 0 and (counts == spp).all()
    err = relative_error(sums.astype(np.float64), expected)
    assert (err <= RELATIVE_TOLERANCE).mean() >= 1.0 - DIVERGED_FRACTION
    # a different sampler: a different image of the same mean
    assert not np.array_equal(sums, hash_sums)
    owen_mean, hash_mean = sums[..., :3].mean(), hash_sums[..., :3].mean()
    assert abs(owen_mean - hash_mean) <= 0.05 * hash_mean


def test_owen_sobol_depth_bound_is_enforced(ctx):
    builder, options, _ = scenes.build_workload("cornell_plain_64")
    options.sampler = OWEN
    options.depth_limits[0] = options.depth_limits[1] = options.depth_limits[2] = 100
    scene = ctx.create_scene(builder)
    inputs = (abi.PathInput * 1)()
    with pytest.raises(runtime.Bf200Error) as info:
        ctx.trace_paths(scene, inputs, options)
    assert info.value.status == 5
    scene.close()
