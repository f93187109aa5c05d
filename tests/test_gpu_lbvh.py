"""The device BLAS build (bf200_context_set_build_mode(BF200_BUILD_DEVICE_LBVH), csrc/bf200_lbvh.cu)
against the host binned-SAH build of the same scene.

Any conservative BVH yields the same closest hit (ties go to the lower instance, then primitive),
so the two builds must agree bit for bit on:
* closest hits (identifiers, t, barycentrics) and occlusion answers of rays aimed at triangle
  edges, vertices and centroids of the BVH-stress scene's meshes;
* a film of the BVH-stress view (320 x 180, 2 spp);
* the edge-ray scene of tests/test_gpu_edges.py with a large mesh added, against the oracle.
The statistics must show the large geometries built on the device.
"""
import os

import numpy as np
import pytest

from bf200 import abi, runtime, scenes
from helpers import bit_equal, sensor_from_golden
from oracle.bindings import Oracle
from test_gpu_edges import edge_rays, edge_scene, ray_array

pytestmark = pytest.mark.gpu


def hit_table(hits):
    ids = np.array([(h.instance_index, h.primitive_index, h.status) for h in hits], np.uint32)
    values = np.array([[h.t] + list(h.barycentrics) for h in hits], np.float32)
    return ids, values


def scene_rays(builder, n, seed):
    """Edge, vertex and centroid rays at the instanced meshes, in world space."""
    rng = np.random.default_rng(seed)
    origins, directions, limits = [], [], []
    per = max(1, n // len(builder.instances))
    for mesh_index, _, matrix, _ in builder.instances:
        mesh = builder.meshes[mesh_index]
        if getattr(mesh, "triangles", None) is None or len(mesh.triangles) == 0:
            continue
        o, d, dist = edge_rays(mesh, per, int(rng.integers(1 << 30)))
        m = np.asarray(matrix, np.float64)
        origins.append((o.astype(np.float64) @ m[:3, :3].T + m[:3, 3]).astype(np.float32))
        directions.append((d.astype(np.float64) @ m[:3, :3].T).astype(np.float32))
        limits.append(np.where(rng.random(len(o)) < 0.5, np.inf, dist * 1.0001).astype(np.float32))
    return np.concatenate(origins), np.concatenate(directions), np.concatenate(limits)


@pytest.fixture(scope="module")
def stress():
    builder, options, _ = scenes.build_workload("bvh_stress_1080p")
    return builder, options


def test_device_build_gives_the_host_builds_hits(stress):
    builder, _ = stress
    origin, direction, t_max = scene_rays(builder, 60000, 3)
    rays = ray_array(origin, direction, t_max)
    with runtime.Context(0, path_capacity=1 << 16) as ctx:
        host = ctx.create_scene(builder)
        ctx.set_build_mode(abi.BUILD_DEVICE_LBVH)
        device = ctx.create_scene(builder)
        hs, ds = host.stats(), device.stats()
        assert hs.device_built_geometries == 0 and ds.device_built_geometries >= 1
        assert ds.leaf_triangle_count == hs.leaf_triangle_count
        h_ids, h_values = hit_table(ctx.closest_hits(host, rays))
        d_ids, d_values = hit_table(ctx.closest_hits(device, rays))
        assert (h_ids[:, 2] == 0).all() and (d_ids[:, 2] == 0).all()
        assert (h_ids == d_ids).all(), f"{(h_ids != d_ids).any(axis=1).sum()} hits differ"
        assert bit_equal(h_values, d_values).all()
        assert (h_ids[:, 0] != 0xFFFFFFFF).mean() > 0.3
        assert (ctx.occlusions(host, rays) == ctx.occlusions(device, rays)).all()
        print(f"host build {hs.total_ms:.1f} ms (BLAS {hs.blas_build_ms:.1f}), device build {ds.total_ms:.1f} ms "
              f"(BLAS {ds.blas_build_ms:.1f}); nodes {hs.node_count} / {ds.node_count}")
        host.close()
        device.close()


def test_device_built_film_is_bit_identical(stress):
    builder, options = stress
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cornell_plain_64.npz"))
    sensor = sensor_from_golden(g)
    origin, normal, tangent, vfov = scenes.workload_camera("bvh_stress_1080p")
    cam = runtime.camera_create(origin, normal, tangent, 320, 180, vfov, scenes.PATH_TIME)
    films = []
    with runtime.Context(0, path_capacity=1 << 18) as ctx:
        for mode in (abi.BUILD_HOST_SAH, abi.BUILD_DEVICE_LBVH):
            ctx.set_build_mode(mode)
            scene = ctx.create_scene(builder)
            sums, counts, _ = ctx.render_film(scene, cam, sensor, options, 2, seed=5)
            films.append(sums)
            scene.close()
    assert bit_equal(films[0], films[1]).all()
    assert films[0][..., :3].sum() > 0.0


def test_device_build_on_the_edge_scene_matches_the_oracle():
    builder, _ = edge_scene()
    big = scenes.displaced_icosphere(5, 0.05, 11)  # 20,480 triangles: above the device-build minimum
    builder.add_instance(builder.add_mesh(big), builder.add_material(scenes.lambertian([0.3] * 4)))
    origin, direction, distance = edge_rays(big, 8000, 9)
    oracle = Oracle(device_trig=True)
    handle = oracle.scene(builder)
    with runtime.Context(0, path_capacity=1 << 16) as ctx:
        ctx.set_build_mode(abi.BUILD_DEVICE_LBVH)
        scene = ctx.create_scene(builder)
        assert scene.stats().device_built_geometries == 1
        for t_max in (np.full(len(origin), np.inf, np.float32), (distance * np.float32(1.0001)).astype(np.float32)):
            rays = ray_array(origin, direction, t_max)
            e_ids, e_values = hit_table(oracle.closest_hits(handle, rays))
            g_ids, g_values = hit_table(ctx.closest_hits(scene, rays))
            assert (e_ids[:, :2] == g_ids[:, :2]).all()
            assert bit_equal(e_values, g_values).all()
        scene.close()
    oracle.destroy(handle)


def test_build_mode_is_checked():
    with runtime.Context(0, path_capacity=1 << 12) as ctx:
        with pytest.raises(runtime.Bf200Error):
            ctx.set_build_mode(7)
