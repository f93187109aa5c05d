"""Writes tests/golden/layered.npz: the reference's own trace_scene_mis (compiled into
oracle/_ref/libbfref.so by `make -C oracle ref`) on the cornell_layered_256 workload -- every
closure kind (Lambert, energy-preserving Oren-Nayar, GGX conductor, GGX dielectric, specular
reflection, specular transmission), multi-closure mixtures with explicit component probabilities,
the ceiling mesh light and a point, a spot and a directional light -- for 1,024 random
(pixel, sample) paths, power MIS, depth 16, Russian roulette from depth 3, with the reference
camera's primary rays.

Run from the repository root: python tests/golden/make_layered_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "blackframe-renderer_b200"))
sys.path.insert(0, os.path.join(REPO, "tests"))

from bf200 import abi, scenes  # noqa: E402
from helpers import arrays  # noqa: E402
from oracle.bindings import Reference  # noqa: E402

WORKLOAD = "cornell_layered_256"
PATHS = 1024


def sample_table(rng, n, width, height, spp):
    return np.stack([rng.integers(0, width, n), rng.integers(0, height, n), rng.integers(0, spp, n),
                     np.zeros(n, np.int64)], axis=1).astype(np.uint64)


def inputs_from(reference, table):
    """PathInputs of a sample table with the reference camera's primary rays."""
    _, _, (width, height, _) = scenes.build_workload(WORKLOAD)
    n = len(table)
    samples = (abi.SampleIndex * n)()
    for k in range(n):
        samples[k].pixel_x, samples[k].pixel_y = int(table[k, 0]), int(table[k, 1])
        samples[k].sample_index, samples[k].seed = int(table[k, 2]), int(table[k, 3])
    rays = reference.camera_rays(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME,
                                 samples)
    inputs = (abi.PathInput * n)()
    for k in range(n):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    return inputs


def terminal(results):
    return np.array([list(r.terminal_ray.origin) + list(r.terminal_ray.direction) for r in results], np.float32)


def main():
    builder, options, (width, height, spp) = scenes.build_workload(WORKLOAD)
    reference = Reference()
    table = sample_table(np.random.default_rng(20261206), PATHS, width, height, spp)
    inputs = inputs_from(reference, table)
    handle = reference.scene(builder)
    results, failures = reference.trace(handle, inputs, options)
    reference.destroy(handle)
    a = arrays(results)
    counters = np.array([list(r.depth_counters) for r in results], np.uint32)
    flags = np.array([r.delta_flags for r in results], np.uint32)
    print(f"{failures} failed paths; {(counters[:, 2] > 0).sum()} with specular bounces, "
          f"{(a['termination'] == 0).sum()} escaped")
    np.savez_compressed(os.path.join(HERE, "layered.npz"), samples=table, radiance=a["radiance"], beta=a["beta"],
                        depth=a["depth"], termination=a["termination"], lane_status=a["lane_status"], eta=a["eta"],
                        depth_counters=counters, delta_flags=flags, terminal=terminal(results))


if __name__ == "__main__":
    main()
