"""Primary rays on the device (bf200_camera_rays: PinholeCamera::generate_primary_ray with the
camera's pixel jitter, PinholeCamera.hpp:144-283, PixelJitter.hpp:47-64) against the oracle's camera,
which tests/test_oracle_golden.py pins on the reference's own rays. The device runs the code that
starts film paths (start_path), so film renders begin from these rays.

Bit for bit, on random pixels and the four corners, sample indices up to 2^40 and random seeds,
centred and jittered, with the hash stream and with Owen-scrambled Sobol."""
import numpy as np
import pytest

from bf200 import abi, runtime, scenes
from oracle.bindings import Oracle

pytestmark = pytest.mark.gpu


def records(width, height, n, seed):
    rng = np.random.default_rng(seed)
    samples = (abi.SampleIndex * n)()
    corners = [(0, 0), (width - 1, 0), (0, height - 1), (width - 1, height - 1)]
    for k in range(n):
        px, py = corners[k] if k < 4 else (int(rng.integers(width)), int(rng.integers(height)))
        samples[k].pixel_x, samples[k].pixel_y = px, py
        samples[k].sample_index = int(rng.integers(1 << 40)) if k % 3 else int(rng.integers(64))
        samples[k].seed = int(rng.integers(1 << 62)) if k % 5 == 0 else 0
    return samples


@pytest.mark.parametrize("workload", ["bvh_stress_1080p", "cornell_spheres_256"])
@pytest.mark.parametrize("sampler", [0, 1])
@pytest.mark.parametrize("jitter", [0, 1])
def test_device_camera_rays_equal_the_oracle(workload, sampler, jitter):
    width, height = scenes.WORKLOADS[workload][:2]
    origin, normal, tangent, vfov = scenes.workload_camera(workload)
    cam = runtime.camera_create(origin, normal, tangent, width, height, vfov, scenes.PATH_TIME, jitter)
    samples = records(width, height, 20000, 17 + sampler + 2 * jitter)
    with runtime.Context(0, path_capacity=1 << 12) as ctx:
        got, status = ctx.camera_rays(cam, samples, sampler)
    expected = Oracle().camera_rays(cam, samples, sampler)
    assert (status == 0).all()
    g = np.frombuffer(bytes(got), np.uint8).reshape(len(samples), -1)
    e = np.frombuffer(bytes(expected), np.uint8).reshape(len(samples), -1)
    differ = (g != e).any(axis=1)
    assert not differ.any(), f"{differ.sum()} of {len(samples)} rays differ"
