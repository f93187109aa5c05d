"""Rays aimed at triangle edges and vertices, from near and far origins.

These rays put the edge functions of the triangle test within rounding of zero: the single-precision
pre-test must pass every such case on to the double-precision test, and the double-precision test
to the exact one, so that hit identifiers, parameters and barycentrics stay bit-exact with the
oracle's exact test (Triangle.hpp:683-822 semantics: shared edges and vertices resolved by the
exact signs, ties by (instance, primitive) order). Occlusion queries over [0, t_max] must agree
with the closest hit's existence.
"""
import numpy as np
import pytest

from bf200 import abi, runtime, scenes
from helpers import bit_equal
from oracle.bindings import Oracle

pytestmark = pytest.mark.gpu


def edge_scene():
    builder = scenes.SceneBuilder(environment=(0.5, 0.5, 0.5, 0.5))
    mesh = scenes.displaced_icosphere(3, 0.05, 7)
    builder.add_instance(builder.add_mesh(mesh), builder.add_material(scenes.lambertian([0.5] * 4)))
    light = builder.add_mesh(scenes.grid_quad((0.0, 0.0), 2.0, 2, 3.0))
    builder.add_instance(light, builder.add_material(scenes.lambertian([0.0] * 4), emission=(1.0, 1.0, 1.0, 1.0)))
    return builder, mesh


def edge_rays(mesh, n, seed):
    rng = np.random.default_rng(seed)
    p = mesh.positions.astype(np.float32)
    tri = mesh.triangles[rng.integers(0, len(mesh.triangles), n)]
    kind = rng.integers(0, 3, n)  # 0 edge point, 1 vertex, 2 centroid
    a = p[tri[:, 0]]
    b = p[tri[:, 1]]
    c = p[tri[:, 2]]
    s = rng.uniform(0.0, 1.0, (n, 1)).astype(np.float32)
    target = np.where((kind == 0)[:, None], (a + s * (b - a)).astype(np.float32), a)
    target = np.where((kind == 2)[:, None], ((a + b + c) / np.float32(3.0)).astype(np.float32), target)
    direction = rng.normal(size=(n, 3))
    direction /= np.linalg.norm(direction, axis=1, keepdims=True)
    direction = direction.astype(np.float32)
    distance = np.float32(10.0) ** rng.integers(-1, 4, n).astype(np.float32)
    origin = (target - distance[:, None] * direction).astype(np.float32)
    return origin, direction, distance


def ray_array(origin, direction, t_max):
    rays = (abi.Ray * len(origin))()
    for k in range(len(origin)):
        for i in range(3):
            rays[k].origin[i], rays[k].direction[i] = float(origin[k, i]), float(direction[k, i])
        rays[k].t_min, rays[k].t_max, rays[k].time, rays[k].mask = 0.0, float(t_max[k]), 0.5, 0xFFFFFFFF
    return rays


def test_edge_and_vertex_rays_bit_exact():
    builder, mesh = edge_scene()
    origin, direction, distance = edge_rays(mesh, 6000, 5)
    oracle = Oracle(device_trig=True)
    handle = oracle.scene(builder)
    with runtime.Context(0, path_capacity=1 << 16) as ctx:
        scene = ctx.create_scene(builder)
        for t_max in (np.full(len(origin), np.inf, np.float32), (distance * np.float32(1.0001)).astype(np.float32)):
            rays = ray_array(origin, direction, t_max)
            expected = oracle.closest_hits(handle, rays)
            got = ctx.closest_hits(scene, rays)
            occluded = ctx.occlusions(scene, rays)
            assert (np.array([h.status for h in got]) == 0).all()
            e_ids = np.array([(h.instance_index, h.primitive_index) for h in expected], np.uint32)
            g_ids = np.array([(h.instance_index, h.primitive_index) for h in got], np.uint32)
            mismatched = (e_ids != g_ids).any(axis=1)
            assert not mismatched.any(), f"{mismatched.sum()} hit-ID mismatches"
            e_t = np.array([[h.t] + list(h.barycentrics) for h in expected], np.float32)
            g_t = np.array([[h.t] + list(h.barycentrics) for h in got], np.float32)
            assert bit_equal(e_t, g_t).all()
            found = e_ids[:, 0] != 0xFFFFFFFF
            assert found.sum() > len(origin) // 4
            assert (occluded == found.astype(np.uint32)).all(), \
                f"{(occluded != found).sum()} occlusion answers differ from the closest hits"
        scene.close()
    oracle.destroy(handle)
