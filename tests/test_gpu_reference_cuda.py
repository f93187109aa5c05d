"""bf200 against the reference's own CUDA backend (oracle/_ref/libbfrefcuda.so: the reference's
XPU/CUDA and Backends/GPU/CUDA sources compiled unchanged for sm_100a by oracle/Makefile).

* Closest hits: instance and primitive identifiers against trace_cuda_closest_hits
  (scene_closest_hit_kernel, CudaSceneClosestHit.cu:1199) on 20,000 rays into each Cornell scene
  and into the 985k-triangle BVH-stress scene. bf200 follows the reference's scalar path bit for
  bit (tests/test_gpu_parity.py); where the reference's CUDA traversal reports another hit, the
  scalar reference is shown to agree with bf200, and such rays stay below 0.5 %. Distances and
  barycentrics are reported, not required: the CUDA traversal rounds them its own way.
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


def scalar_hits(builder):
    """Closest hits of the oracle restatement (pinned on the reference's scalar path) for a subset."""
    def run(rays):
        oracle = Oracle()
        handle = oracle.scene(builder)
        hits = oracle.closest_hits(handle, rays)
        oracle.destroy(handle)
        return hits
    return run


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


def hit_arrays(hits):
    ids = np.array([(h.instance_index, h.primitive_index) for h in hits], np.uint32)
    tb = np.array([[h.t] + list(h.barycentrics) for h in hits], np.float32)
    return ids, tb


def compare_hits(expected, got, label, rays, oracle_hits):
    """Hit identifiers of bf200 against the reference CUDA traversal. Where the two differ, bf200
    must agree with the reference's scalar path (the oracle restatement, pinned bit-exact on the
    compiled reference), i.e. the difference is one between the reference's own two backends."""
    e_ids, e_tb = hit_arrays(expected)
    g_ids, g_tb = hit_arrays(got)
    assert (np.array([h.status for h in got]) == 0).all()
    assert (e_ids[:, 0] != 0xFFFFFFFF).sum() > len(expected) // 5
    mismatch = (e_ids != g_ids).any(axis=1)
    hit = (e_ids[:, 0] != 0xFFFFFFFF) & ~mismatch
    same_tb = bit_equal(e_tb[hit], g_tb[hit]).all(axis=1)
    print(f"{label}: {len(expected) - mismatch.sum()}/{len(expected)} hit identifiers equal to the reference CUDA "
          f"traversal; distance and barycentrics bit-exact on {same_tb.sum()}/{hit.sum()} common hits")
    if mismatch.any():
        index = np.nonzero(mismatch)[0]
        sub = (abi.Ray * len(index))(*[rays[k] for k in index])
        o_ids, o_tb = hit_arrays(oracle_hits(sub))
        for j, k in enumerate(index[:6]):
            print(f"  ray {k}: reference CUDA {tuple(e_ids[k])} t={e_tb[k, 0]!r}, bf200 {tuple(g_ids[k])} "
                  f"t={g_tb[k, 0]!r}, scalar reference {tuple(o_ids[j])} t={o_tb[j, 0]!r}")
        assert (o_ids == g_ids[index]).all(), f"{label}: bf200 differs from the scalar reference where the CUDA one does"
        assert bit_equal(o_tb, g_tb[index]).all()
    assert mismatch.mean() <= 0.005, f"{label}: {mismatch.sum()} hit-ID mismatches"


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
    compare_hits(expected, got, name, rays, scalar_hits(builder))


def test_bvh_stress_hit_ids_bit_exact_against_reference_cuda(ctx, refcuda):
    builder, _, _ = scenes.build_workload("bvh_stress_1080p")
    rays = random_rays(20000, 21, -14.0, 14.0)
    handle = refcuda.scene(builder)
    expected = refcuda.closest_hits(handle, rays)
    refcuda.destroy(handle)
    scene = ctx.create_scene(builder)
    got = ctx.closest_hits(scene, rays)
    scene.close()
    compare_hits(expected, got, "bvh_stress_1080p", rays, scalar_hits(builder))


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
