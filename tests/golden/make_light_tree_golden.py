"""Writes tests/golden/light_tree.npz: the reference's spatial light tree
(LightSampler::create_spatial_tree, compiled into oracle/_ref/libbfref.so by `make -C oracle ref`)
on seeded light sets: for query points inside, near and far from the lights, the selection of
canonical samples (slot and probability) and the probability of every light.

The sets cover one light, clustered and spread boxes, flat and point-like boxes, zero-power
lights, canonically unbounded lights beside finite ones and alone, and coincident centroids.

Run from the repository root: python tests/golden/make_light_tree_golden.py, and with the argument
`transport` for tests/golden/light_tree_transport.npz: the reference's trace_scene_mis selecting
by the tree on a three-light Cornell box.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "blackframe-renderer_b200"))

from oracle.bindings import Reference  # noqa: E402

INF = np.float32(np.inf)


def light_sets(rng):
    sets = []

    def boxes(n, spread, size):
        centre = rng.uniform(-spread, spread, (n, 3))
        half = rng.uniform(0.0, size, (n, 3))
        return (centre - half).astype(np.float32), (centre + half).astype(np.float32)

    def powers(n, zero_share=0.0):
        p = rng.lognormal(0.0, 1.5, (n, 4)).astype(np.float32)
        p[rng.random(n) < zero_share] = 0.0
        return p

    lo, hi = boxes(1, 1.0, 0.5)
    sets.append((lo, hi, powers(1)))                                   # one light
    for n, spread, size in ((2, 1.0, 0.2), (7, 5.0, 1.0), (64, 20.0, 0.5), (300, 100.0, 3.0)):
        lo, hi = boxes(n, spread, size)
        sets.append((lo, hi, powers(n, 0.1)))
    lo, hi = boxes(16, 3.0, 0.0)                                        # point-like boxes
    sets.append((lo, hi, powers(16)))
    lo, hi = boxes(16, 3.0, 1.0)
    lo[:, 1] = hi[:, 1] = np.float32(2.0)                               # flat boxes at one height
    sets.append((lo, hi, powers(16)))
    lo, hi = boxes(12, 4.0, 0.5)                                        # unbounded lights mixed in
    lo[[2, 7, 9]] = -INF
    hi[[2, 7, 9]] = INF
    sets.append((lo, hi, powers(12)))
    lo = np.full((3, 3), -INF, np.float32)                              # unbounded lights alone
    hi = np.full((3, 3), INF, np.float32)
    sets.append((lo, hi, powers(3)))
    lo, hi = boxes(1, 1.0, 0.5)                                         # coincident centroids
    lo, hi = np.repeat(lo, 9, axis=0), np.repeat(hi, 9, axis=0)
    sets.append((lo, hi, powers(9)))
    return sets


def queries(rng, lo, hi, n):
    finite = np.isfinite(lo).all(axis=1)
    if finite.any():
        centre = (lo[finite] + hi[finite]) / 2
        scale = float(np.abs(centre).max()) + 1.0
    else:
        centre, scale = np.zeros((1, 3)), 1.0
    picks = centre[rng.integers(0, len(centre), n)]
    near = picks + rng.normal(0.0, 0.3, (n, 3))
    far = rng.uniform(-10 * scale, 10 * scale, (n, 3))
    positions = np.where((rng.random(n) < 0.5)[:, None], near, far).astype(np.float32)
    positions[0] = picks[0]  # inside a light's box
    samples = rng.random(n).astype(np.float32)
    samples[:4] = [0.0, 0.5, np.nextafter(np.float32(1.0), np.float32(0.0)), 1e-9]
    return positions, samples


def main():
    ref = Reference()
    rng = np.random.default_rng(20261206)
    out = {}
    sets = light_sets(rng)
    for k, (lo, hi, p) in enumerate(sets):
        positions, samples = queries(rng, lo, hi, 256)
        picked, code = ref.light_tree(lo, hi, p, positions, samples=samples)
        assert code == 0, (k, code)
        selected, probabilities = picked
        # the probability of every light at the first 32 points
        grid = np.repeat(positions[:32], len(p), axis=0)
        indices = np.tile(np.arange(len(p), dtype=np.uint32), 32)
        each, code = ref.light_tree(lo, hi, p, grid, light_indices=indices)
        assert code == 0, (k, code)
        out.update({f"lo_{k}": lo, f"hi_{k}": hi, f"powers_{k}": p, f"positions_{k}": positions,
                    f"samples_{k}": samples, f"selected_{k}": selected, f"probability_{k}": probabilities,
                    f"each_{k}": each[1].reshape(32, len(p))})
    out["sets"] = np.int64(len(sets))
    np.savez_compressed(os.path.join(HERE, "light_tree.npz"), **out)
    print(f"{len(sets)} light sets written")


def tree_box_inputs(builder):
    """bf200_light_tree_input_v1 per emissive instance of a builder (registry order): the world
    bounds of its mesh and its flux per lane (radiance x area x pi)."""
    sys.path.insert(0, os.path.dirname(HERE))
    from bf200 import abi
    from test_gpu_light_power import light_powers
    powers = light_powers(builder)
    lights = (abi.LightTreeInput * len(powers))()
    k = 0
    for mesh_index, material, to_world, _ in builder.instances:
        if not any(v != 0 for v in builder.materials[material][1]):
            continue
        m = np.asarray(to_world, np.float64).reshape(4, 4)
        p = np.asarray(builder.meshes[mesh_index].positions, np.float64)
        world = (p @ m[:3, :3].T + m[:3, 3]).astype(np.float32)
        lights[k].bounds_min[:] = [float(v) for v in world.min(axis=0)]
        lights[k].bounds_max[:] = [float(v) for v in world.max(axis=0)]
        lights[k].spectral_power[:] = [float(v) for v in powers[k]]
        k += 1
    return lights


def transport():
    """The reference's trace_scene_mis with the spatial light tree on the three-light box:
    tests/golden/light_tree_transport.npz."""
    sys.path.insert(0, os.path.dirname(HERE))
    from bf200 import abi
    from oracle.bindings import Oracle
    from test_gpu_light_power import path_inputs, three_light_box
    builder = three_light_box()
    lights = tree_box_inputs(builder)
    inputs = path_inputs(Oracle(), 512, 23)
    options = abi.default_options(mis="power", max_depth=8)
    ref = Reference()
    h = ref.scene(builder)
    ref.set_light_tree(h, lights)
    results, failures = ref.trace(h, inputs, options)
    ref.destroy(h)
    np.savez_compressed(os.path.join(HERE, "light_tree_transport.npz"),
                        radiance=np.array([list(r.radiance) for r in results], np.float32),
                        beta=np.array([list(r.beta) for r in results], np.float32),
                        depth=np.array([r.depth for r in results], np.uint32),
                        termination=np.array([r.termination for r in results], np.uint32),
                        lane_status=np.array([r.lane_status for r in results], np.uint32))
    print(f"tree transport: 512 paths, {failures} refused")


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "transport":
        transport()
    else:
        main()
