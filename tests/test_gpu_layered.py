"""Closure mixtures, rough diffuse and specular closures and punctual lights on the device: the
cornell_layered_256 workload (every closure kind; layered Lambert + GGX conductor and specular
reflection + transmission mixtures with explicit component probabilities; a point, a spot and a
directional light beside the ceiling mesh light) against the oracle, whose results on this scene
are pinned bit for bit on the compiled reference by tests/test_closure_mixtures.py. The oracle
rounds sampled-angle sines and cosines as the device does (device_trig)."""
import os

import numpy as np
import pytest

from bf200 import abi, runtime, scenes
from helpers import arrays, bit_equal, check_paths, relative_error, sensor_from_golden, RELATIVE_TOLERANCE
from oracle.bindings import Oracle

pytestmark = pytest.mark.gpu
NAME = "cornell_layered_256"


@pytest.fixture(scope="module")
def ctx():
    with runtime.Context(0, path_capacity=1 << 16) as c:
        yield c


@pytest.fixture(scope="module")
def workload():
    builder, options, (width, height, spp) = scenes.build_workload(NAME)
    rng = np.random.default_rng(99)
    n = 8192
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    samples = (abi.SampleIndex * n)()
    for k in range(n):
        samples[k].pixel_x, samples[k].pixel_y = int(rng.integers(width)), int(rng.integers(height))
        samples[k].sample_index, samples[k].seed = int(rng.integers(1 << 40)), 0x243F6A8885A308D3
    oracle = Oracle(device_trig=True)
    rays = oracle.camera_rays(cam, samples)
    inputs = (abi.PathInput * n)()
    for k in range(n):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    return builder, options, inputs, cam


def test_layered_paths_match_the_oracle(ctx, workload):
    builder, options, inputs, _ = workload
    oracle = Oracle(device_trig=True)
    handle = oracle.scene(builder)
    expected, failures = oracle.trace(handle, inputs, options)
    oracle.destroy(handle)
    scene = ctx.create_scene(builder)
    got, report = ctx.trace_paths(scene, inputs, options)
    scene.close()
    a, b = arrays(got), arrays(expected)
    assert np.array_equal(a["lane_status"] != 0, b["lane_status"] != 0)
    keep = b["lane_status"] == 0
    exact, close = check_paths({k: v[keep] for k, v in a.items()}, {k: v[keep] for k, v in b.items()}, NAME,
                               diverged=0.0)
    assert exact >= 0.99
    # every output of a bit-exact path is identical: depth counters, delta flags, eta scale
    same = bit_equal(a["radiance"], b["radiance"]).all(axis=1) & keep
    for k in np.nonzero(same)[0][:2048]:
        assert bytes(got[k]) == bytes(expected[k]), k
    counters = np.array([list(r.depth_counters) for r in got], np.uint32)
    flags = np.array([r.delta_flags for r in got], np.uint32)
    assert (counters[:, 2] > 0).sum() > 200 and ((flags & 1) != 0).sum() > 50  # specular chains ran


def test_layered_cones_match_the_oracle(ctx, workload):
    builder, options, inputs, _ = workload
    n = 4096
    sub = (abi.PathInput * n)(*inputs[:n])
    cones = np.tile(np.array([0.0, 0.0015], np.float32), (n, 1))
    oracle = Oracle(device_trig=True)
    handle = oracle.scene(builder)
    expected, expected_cones, _ = oracle.trace_cones(handle, sub, cones, options)
    oracle.destroy(handle)
    scene = ctx.create_scene(builder)
    got, got_cones, report = ctx.trace_paths_with_cones(scene, sub, cones, options)
    scene.close()
    a, b = arrays(got), arrays(expected)
    assert np.array_equal(a["lane_status"] != 0, b["lane_status"] != 0)
    keep = b["lane_status"] == 0
    check_paths({k: v[keep] for k, v in a.items()}, {k: v[keep] for k, v in b.items()}, NAME + " with cones",
                diverged=0.0)
    same = bit_equal(a["radiance"], b["radiance"]).all(axis=1) & keep
    assert bit_equal(got_cones, expected_cones).all(axis=1)[same].mean() >= 0.999
    assert (relative_error(got_cones, expected_cones) <= RELATIVE_TOLERANCE).all(axis=1)[keep].mean() >= 0.999


def test_layered_film_matches_the_oracle(ctx, workload):
    builder, options, _, _ = workload
    width, height, spp = 48, 48, 4
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cornell_spheres_256.npz"))
    sensor = sensor_from_golden(g)
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    scene = ctx.create_scene(builder)
    sums, counts, report = ctx.render_film(scene, cam, sensor, options, spp, seed=0, precision=1)
    scene.close()
    oracle = Oracle(device_trig=True)
    px, py, s = np.meshgrid(np.arange(width), np.arange(height), np.arange(spp), indexing="ij")
    order = np.lexsort((px.ravel(), py.ravel(), s.ravel()))
    px, py, s = px.ravel()[order], py.ravel()[order], s.ravel()[order]
    samples = (abi.SampleIndex * len(px))()
    for k in range(len(px)):
        samples[k].pixel_x, samples[k].pixel_y, samples[k].sample_index = int(px[k]), int(py[k]), int(s[k])
    rays = oracle.camera_rays(cam, samples)
    inputs = (abi.PathInput * len(px))()
    for k in range(len(px)):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    handle = oracle.scene(builder)
    results, failures = oracle.trace(handle, inputs, options)
    oracle.destroy(handle)
    expected, _ = oracle.film(arrays(results)["radiance"], samples, sensor, width, height, 1)
    got = sums[..., :4] + sums[..., 4:]
    assert report.failed_lanes == failures
    assert (relative_error(got, expected) <= RELATIVE_TOLERANCE).all()


def test_punctual_only_scene(ctx):
    """A scene lit by a point light alone (no mesh light): the registry is the punctual light."""
    builder = scenes.SceneBuilder()
    white = builder.add_material(scenes.lambertian([0.6] * 4))
    builder.add_instance(builder.add_mesh(scenes.quad([(-1, -1, 0), (-1, -1, 2), (1, -1, 2), (1, -1, 0)],
                                                      (0, 1, 0))), white)
    builder.add_point_light((0.0, 0.5, 1.0), (1.0, 1.0, 1.0, 1.0))
    options = abi.default_options(mis="power", max_depth=4)
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), 16, 16, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    samples = (abi.SampleIndex * 256)()
    for k in range(256):
        samples[k].pixel_x, samples[k].pixel_y = k % 16, k // 16
    oracle = Oracle(device_trig=True)
    rays = oracle.camera_rays(cam, samples)
    inputs = (abi.PathInput * 256)()
    for k in range(256):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    handle = oracle.scene(builder)
    expected, _ = oracle.trace(handle, inputs, options)
    oracle.destroy(handle)
    scene = ctx.create_scene(builder)
    got, report = ctx.trace_paths(scene, inputs, options)
    scene.close()
    assert report.registered_light_count == 1
    a, b = arrays(got), arrays(expected)
    assert (a["radiance"] > 0).any(axis=1).sum() > 20
    check_paths(a, b, "point light only", diverged=0.0)


def test_invalid_punctual_lights_are_refused(ctx):
    for light in [dict(kind="spot", inner=0.7, outer=0.5), dict(kind="directional", direction=(0.0, 0.0, 2.0))]:
        builder, _, _ = scenes.build_workload("cornell_plain_64")
        if light["kind"] == "spot":
            builder.add_spot_light((0.0, 0.5, 1.0), (0.0, -1.0, 0.0), light["inner"], light["outer"], (1.0,) * 4)
        else:
            builder.add_directional_light(light["direction"], (1.0,) * 4)
        with pytest.raises(runtime.Bf200Error) as info:
            ctx.create_scene(builder)
        assert info.value.status == 1
