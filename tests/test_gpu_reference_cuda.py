"""bf200 against the reference's own CUDA backend (oracle/_ref/libbfrefcuda.so: the reference's
XPU/CUDA and Backends/GPU/CUDA sources compiled unchanged for sm_100a by oracle/Makefile).

* Closest hits: instance and primitive identifiers, hit distance and barycentrics bit-exact
  against trace_cuda_closest_hits (scene_closest_hit_kernel, CudaSceneClosestHit.cu:1199) on
  20,000 rays into each Cornell scene and into the 985k-triangle BVH-stress scene.
* Transport: per-path results of bf200_trace_paths_with_cones against
  trace_cuda_wavefront_transport on the same inputs (primary rays and cones of the reference
  camera, PathState::create_initial, the same sample indices).
"""
import numpy as np
import pytest

from bf200 import abi, runtime, scenes
from helpers import arrays, bit_equal, relative_error, RELATIVE_TOLERANCE
from oracle.bindings import Oracle, ReferenceCuda, reference_cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not reference_cuda_available(), reason="oracle/_ref/libbfrefcuda.so not built")]


@pytest.fixture(scope="module")
def ctx():
    with runtime.Context(0, path_capacity=1 << 16) as c:
        yield c


@pytest.fixture(scope="module")
def refcuda():
    return ReferenceCuda()


def random_rays(n, seed, lo, hi, z=None):
    rng = np.random.default_rng(seed)
    origins = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    if z is not None:
        origins[:, 2] = rng.uniform(z[0], z[1], n).astype(np.float32)
    directions = rng.normal(size=(n, 3)).astype(np.float32)
    directions /= np.linalg.norm(directions, axis=1, keepdims=True)
    rays = (abi.Ray * n)()
    for k in range(n):
        for a in range(3):
            rays[k].origin[a], rays[k].direction[a] = float(origins[k, a]), float(directions[k, a])
        rays[k].t_min, rays[k].t_max, rays[k].time, rays[k].mask = 0.0, float("inf"), 0.5, 0xFFFFFFFF
    return rays


def compare_hits(expected, got, label):
    e_ids = np.array([(h.instance_index, h.primitive_index) for h in expected], np.uint32)
    g_ids = np.array([(h.instance_index, h.primitive_index) for h in got], np.uint32)
    assert (np.array([h.status for h in got]) == 0).all()
    mismatch = (e_ids != g_ids).any(axis=1)
    assert not mismatch.any(), f"{label}: {mismatch.sum()} hit-ID mismatches, first {np.nonzero(mismatch)[0][:8]}"
    assert (e_ids[:, 0] != 0xFFFFFFFF).sum() > len(expected) // 5
    e_t = np.array([[h.t] + list(h.barycentrics) for h in expected], np.float32)
    g_t = np.array([[h.t] + list(h.barycentrics) for h in got], np.float32)
    hit = e_ids[:, 0] != 0xFFFFFFFF
    assert bit_equal(e_t[hit], g_t[hit]).all(), f"{label}: {(~bit_equal(e_t[hit], g_t[hit]).all(axis=1)).sum()} distances differ"


@pytest.mark.parametrize("name", ["cornell_plain_64", "cornell_spheres_256"])
def test_hit_ids_bit_exact_against_reference_cuda(ctx, refcuda, name):
    builder, _, _ = scenes.build_workload(name)
    rays = random_rays(20000, 11, -0.99, 0.99, z=(0.01, 3.5))
    handle = refcuda.scene(builder)
    expected = refcuda.closest_hits(handle, rays)
    refcuda.destroy(handle)
    scene = ctx.create_scene(builder)
    got = ctx.closest_hits(scene, rays)
    scene.close()
    compare_hits(expected, got, name)


def test_bvh_stress_hit_ids_bit_exact_against_reference_cuda(ctx, refcuda):
    builder, _, _ = scenes.build_workload("bvh_stress_1080p")
    rays = random_rays(20000, 21, -14.0, 14.0)
    handle = refcuda.scene(builder)
    expected = refcuda.closest_hits(handle, rays)
    refcuda.destroy(handle)
    scene = ctx.create_scene(builder)
    got = ctx.closest_hits(scene, rays)
    scene.close()
    compare_hits(expected, got, "bvh_stress_1080p")


def test_transport_against_reference_cuda(ctx, refcuda, golden):
    """The Cornell box with its conductor and dielectric spheres, 4,096 paths started with the
    reference camera's rays and cones: lane failures and per-path results against the reference
    CUDA wavefront."""
    g = golden("cones")
    builder, options, (width, height, _) = scenes.build_workload("cornell_spheres_256")
    table = g["camera_samples"]
    n = len(table)
    samples = (abi.SampleIndex * n)()
    for k in range(n):
        samples[k].pixel_x, samples[k].pixel_y = int(table[k, 0]), int(table[k, 1])
        samples[k].sample_index, samples[k].seed = int(table[k, 2]), int(table[k, 3])
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    rays = Oracle().camera_rays(cam, samples)
    inputs = (abi.PathInput * n)()
    for k in range(n):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    cones = g["camera_cones"]
    handle = refcuda.scene(builder)
    expected, ref_report, _ = refcuda.trace(handle, inputs, options, cones=cones)
    refcuda.destroy(handle)
    scene = ctx.create_scene(builder)
    results, _, report = ctx.trace_paths_with_cones(scene, inputs, cones, options)
    scene.close()
    got, want = arrays(results), arrays(expected)
    ok = got["lane_status"] == 0
    same = bit_equal(got["radiance"], want["radiance"]).all(axis=1) & ok
    close = (relative_error(got["radiance"], want["radiance"]) <= RELATIVE_TOLERANCE).all(axis=1) & ok
    terminations = (got["termination"] == want["termination"]) & ok
    print(f"reference CUDA: {same.sum()}/{n} bit-exact, {close.sum()}/{n} within {RELATIVE_TOLERANCE}, "
          f"{terminations.sum()}/{n} same termination, bf200 failed {(~ok).sum()}; "
          f"segments bf200 {report.extension_segments}/{report.shadow_segments} "
          f"reference {ref_report.extension_segments}/{ref_report.shadow_segments}")
    assert ref_report.terminated_paths == n
    assert close.mean() >= 0.9 and terminations.mean() >= 0.9
