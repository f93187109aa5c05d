"""The oracle restatement against the reference's own outputs (committed golden fixtures).

The fixtures come from the reference implementation compiled from its sources
(tests/golden/make_golden.py). These tests pin the oracle: bit-exact per-path results, the
committed inverse transforms, the CIE film path and the SampleStream hash.
"""
import numpy as np
import pytest

from bf200 import abi, scenes
from helpers import arrays, bit_equal, golden_inputs, sensor_from_golden
from oracle.bindings import Oracle

WORKLOADS = ["cornell_plain_64", "cornell_spheres_256"]


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


@pytest.mark.parametrize("name", WORKLOADS)
def test_scene_inverse_matches_frame_scene(golden, name):
    g = golden(name)
    builder, _, _ = scenes.build_workload(name)
    desc = builder.desc()
    for i in range(desc.instance_count):
        mine = np.array(desc.instances[i].world_to_object[:], np.float32)
        assert bit_equal(mine, g["world_to_object"][i]).all(), f"instance {i}"


@pytest.mark.parametrize("name", WORKLOADS)
def test_oracle_paths_bit_exact(oracle, golden, name):
    g = golden(name)
    builder, options, _ = scenes.build_workload(name)
    handle = oracle.scene(builder)
    results, failures = oracle.trace(handle, golden_inputs(g), options)
    oracle.destroy(handle)
    assert failures == 0
    got = arrays(results)
    assert bit_equal(got["radiance"], g["radiance"]).all()
    assert bit_equal(got["beta"], g["beta"]).all()
    assert (got["depth"] == g["depth"]).all()
    assert (got["termination"] == g["termination"]).all()
    assert bit_equal(got["eta"], g["eta"]).all()


def camera_from_golden(g, key, width, height):
    c = g[key]
    cam = abi.Camera()
    for a in range(3):
        cam.origin[a], cam.tangent[a] = float(c[a]), float(c[3 + a])
        cam.bitangent[a], cam.normal[a] = float(c[6 + a]), float(c[9 + a])
    cam.half_width, cam.half_height = float(c[12]), float(c[13])
    cam.t_min, cam.t_max, cam.time = 0.0, float("inf"), scenes.PATH_TIME
    cam.mask, cam.width, cam.height, cam.jitter_mode = 0xFFFFFFFF, width, height, 1
    return cam


def film_samples(fw, fh, fspp):
    px, py, s = np.meshgrid(np.arange(fw), np.arange(fh), np.arange(fspp), indexing="ij")
    order = np.lexsort((px.ravel(), py.ravel(), s.ravel()))
    px, py, s = px.ravel()[order], py.ravel()[order], s.ravel()[order]
    samples = (abi.SampleIndex * len(px))()
    for k in range(len(px)):
        samples[k].pixel_x, samples[k].pixel_y, samples[k].sample_index = int(px[k]), int(py[k]), int(s[k])
    return samples


@pytest.mark.parametrize("name", WORKLOADS)
def test_oracle_camera_rays_match_reference(oracle, golden, name):
    g = golden(name)
    _, _, (width, height, _) = scenes.build_workload(name)
    cam = camera_from_golden(g, "camera", width, height)
    n = len(g["pixel_x"])
    samples = (abi.SampleIndex * n)()
    for k in range(n):
        samples[k].pixel_x, samples[k].pixel_y = int(g["pixel_x"][k]), int(g["pixel_y"][k])
        samples[k].sample_index = int(g["sample_index"][k])
    rays = oracle.camera_rays(cam, samples)
    direction = np.array([list(r.direction) for r in rays], np.float32).reshape(n, 3)
    assert bit_equal(direction, g["ray_direction"]).all()


@pytest.mark.parametrize("name", WORKLOADS)
@pytest.mark.parametrize("precision", [0, 1])
def test_oracle_film_matches_reference_film(oracle, golden, name, precision):
    g = golden(name)
    builder, options, _ = scenes.build_workload(name)
    fw, fh, fspp = (int(v) for v in g["film_size"])
    samples = film_samples(fw, fh, fspp)
    rays = oracle.camera_rays(camera_from_golden(g, "film_camera", fw, fh), samples)
    inputs = (abi.PathInput * len(samples))()
    for k in range(len(samples)):
        inputs[k].primary_ray = rays[k]
        inputs[k].sample = samples[k]
    handle = oracle.scene(builder)
    results, failures = oracle.trace(handle, inputs, options)
    oracle.destroy(handle)
    assert failures == 0
    radiance = arrays(results)["radiance"]
    sums, counts = oracle.film(radiance, samples, sensor_from_golden(g), fw, fh, precision)
    expected = g["film32"] if precision == 0 else g["film64"]
    assert (counts == (g["counts32"] if precision == 0 else g["counts64"])).all()
    if precision == 0:
        assert bit_equal(sums.astype(np.float32), expected.astype(np.float32)).all()
    else:
        assert (sums == expected).all()


def test_sample_stream_known_values(oracle):
    # SampleStream.hpp:23-45: mix_bits is the SplitMix64 finaliser; pin a few values computed
    # independently in Python.
    def mix(v):
        m = (1 << 64) - 1
        v ^= v >> 30
        v = (v * 0xBF58476D1CE4E5B9) & m
        v ^= v >> 27
        v = (v * 0x94D049BB133111EB) & m
        return v ^ (v >> 31)

    def sample(px, py, s, seed, dim):
        st = mix(seed ^ 0x9E3779B97F4A7C15)
        st = mix(st ^ ((px << 32) | py) ^ 0xD1B54A32D192ED03)
        st = mix(st ^ s ^ 0x8CB92BA72F3D8DD7)
        return np.float32(mix(st ^ dim) >> 40) * np.float32(2.0 ** -24)

    assert 0.0 <= sample(3, 5, 7, 0, 4) < 1.0
    assert sample(3, 5, 7, 0, 4) != sample(3, 5, 7, 0, 5)
    assert sample(0, 0, 0, 0, 0) == sample(0, 0, 0, 0, 0)
