"""Writes tests/golden/spheres.npz: analytic sphere intersections computed by the reference itself
(renderer::Sphere, Sphere.hpp, compiled into oracle/_ref/libbfref.so by `make -C oracle ref`).

* pair_*: ray k against sphere k. The first rows are the cases of the reference's own
  Tests/Renderer/SphereTest.cpp (near and far roots with closed bounds, excluded roots, the internal
  root of a non-unit direction, a surface origin, double tangents, a distant oblique tangent,
  squared products rounding in opposite directions, a tiny direction, the cardinal normals, a miss
  and an arithmetic error). After them come seeded random rays, origins inside and outside.
* scene_*: 8 seeded spheres and 1,024 rays aimed near them, with every (ray, sphere) result, for
  the closest-hit test of a scene that holds all 8 spheres.

Per result, 8 floats: status (0 miss, 1 hit, 2 the reference reported an error), t, outward
normal xyz, hit position xyz. Run from the repository root: python tests/golden/make_sphere_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "blackframe-renderer_b200"))

from bf200 import abi  # noqa: E402
from oracle.bindings import Reference  # noqa: E402

INF = float("inf")
F32_MAX = float(np.finfo(np.float32).max)


def up(x, toward):
    return float(np.nextafter(np.float32(x), np.float32(toward)))


def reference_cases():
    """(centre xyz, radius, origin xyz, direction xyz, t_min, t_max) from SphereTest.cpp."""
    c = []
    unit = (0.0, 0.0, 0.0, 1.0)
    c.append((*unit, 0.0, 0.0, -3.0, 0.0, 0.0, 1.0, 0.0, INF))             # near root
    c.append((*unit, 0.0, 0.0, -3.0, 0.0, 0.0, 1.0, 3.0, 4.0))             # far root
    c.append((*unit, 0.0, 0.0, -3.0, 0.0, 0.0, 1.0, 2.0, 2.0))             # closed lower bound
    c.append((*unit, 0.0, 0.0, -3.0, 0.0, 0.0, 1.0, 4.0, 4.0))             # closed upper bound
    c.append((*unit, 0.0, 0.0, -3.0, 0.0, 0.0, 1.0, up(2.0, 3.0), up(4.0, 3.0)))  # both excluded
    c.append((*unit, 0.0, 0.0, 0.0, 2.0, 0.0, 0.0, 0.0, INF))              # internal, non-unit d
    c.append((0.0, 0.0, 0.0, 0.1, 0.1, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0))  # surface origin
    c.append((*unit, -2.0, 1.0, 0.0, 1.0, 0.0, 0.0, 2.0, 2.0))             # double tangent
    c.append((0.0, 0.0, 0.0, 5.0, -399997.0, 300004.0, 0.0, 4.0, -3.0, 0.0, 0.0, INF))  # distant tangent
    c.append((0.0, 0.0, 0.0, 149.0, -89.0, 191.0, 0.0, 140.0, -51.0, 0.0, 1.0, 1.0))
    c.append((0.0, 0.0, 0.0, 149.0, -89.0, up(191.0, 192.0), 0.0, 140.0, -51.0, 0.0, 0.0, INF))
    c.append((0.0, 0.0, 0.0, 149.0, -89.0, up(191.0, 190.0), 0.0, 140.0, -51.0, 0.0, 0.0, INF))
    c.append((*unit, 0.0, 0.0, -3.0, 0.0, 0.0, 1.0e-22, 0.0, INF))         # tiny direction
    c.append((1.0, 2.0, 3.0, 5.0, 7.0, 10.0, 3.0, -3.0, -4.0, 0.0, 0.0, INF))  # translated sphere
    for origin, direction in [((3, 0, 0), (-1, 0, 0)), ((0, 0, 3), (0, 0, -1)), ((-3, 0, 0), (1, 0, 0)),
                              ((0, 0, -3), (0, 0, 1)), ((0, 3, 0), (0, -1, 0)), ((0, -3, 0), (0, 1, 0))]:
        c.append((*unit, *map(float, origin), *map(float, direction), 0.0, INF))  # cardinal normals
    c.append((*unit, 0.0, 2.0, -3.0, 0.0, 0.0, 1.0, 0.0, INF))             # miss
    c.append((F32_MAX, 0.0, 0.0, 1.0, -F32_MAX, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, INF))  # arithmetic error
    return c


def random_pairs(rng, n):
    cases = []
    for _ in range(n):
        centre = rng.normal(0.0, 2.0, 3)
        radius = float(np.exp(rng.normal(-1.0, 1.0)))
        origin = centre + rng.normal(0.0, 1.0, 3) * radius * rng.choice([0.5, 2.0, 10.0])
        direction = centre + rng.normal(0.0, 1.0, 3) * radius * 1.2 - origin
        if rng.random() < 0.3:
            direction = direction * rng.uniform(0.1, 10.0)
        t_min = 0.0 if rng.random() < 0.8 else float(rng.uniform(0.0, 2.0))
        cases.append((*centre, radius, *origin, *direction, t_min, INF))
    return cases


def as_inputs(cases):
    a = np.array(cases, np.float64).astype(np.float32)
    spheres = a[:, 0:4]
    rays = (abi.Ray * len(a))()
    for k, row in enumerate(a):
        for i in range(3):
            rays[k].origin[i] = float(row[4 + i])
            rays[k].direction[i] = float(row[7 + i])
        rays[k].t_min, rays[k].t_max = float(row[10]), float(row[11])
        rays[k].time, rays[k].mask = 0.5, 0xFFFFFFFF
    ray_rows = a[:, 4:12]
    return spheres, rays, ray_rows


def main():
    ref = Reference()
    rng = np.random.default_rng(20261203)
    cases = reference_cases() + random_pairs(rng, 4096)
    spheres, rays, ray_rows = as_inputs(cases)
    pair_out = ref.sphere_intersect(spheres, rays)

    scene_spheres = np.zeros((8, 4), np.float32)
    for s in range(8):
        scene_spheres[s, :3] = rng.uniform(-3.0, 3.0, 3)
        scene_spheres[s, 3] = rng.uniform(0.3, 1.2)
    scene_cases = []
    for _ in range(1024):
        target = scene_spheres[rng.integers(8), :3] + rng.normal(0.0, 0.8, 3)
        origin = rng.normal(0.0, 1.0, 3)
        origin = origin / np.linalg.norm(origin) * rng.uniform(6.0, 12.0)
        scene_cases.append((0.0, 0.0, 0.0, 1.0, *origin, *(target - origin), 0.0, INF))
    _, scene_rays, scene_ray_rows = as_inputs(scene_cases)
    scene_out = np.zeros((len(scene_cases), 8, 8), np.float32)
    for s in range(8):
        scene_out[:, s, :] = ref.sphere_intersect(np.repeat(scene_spheres[s:s + 1], len(scene_cases), 0), scene_rays)
    np.savez_compressed(os.path.join(HERE, "spheres.npz"), pair_spheres=spheres, pair_rays=ray_rows, pair_out=pair_out,
                        reference_cases=np.int64(len(reference_cases())), scene_spheres=scene_spheres,
                        scene_rays=scene_ray_rows, scene_out=scene_out)
    status, counts = np.unique(pair_out[:, 0], return_counts=True)
    print("pairs:", dict(zip(status.tolist(), counts.tolist())), "scene hits:", int((scene_out[:, :, 0] == 1).sum()))


if __name__ == "__main__":
    main()
