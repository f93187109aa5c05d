"""Writes tests/golden/initial_states.npz: the reference's own trace_scene_mis (compiled into
oracle/_ref/libbfref.so by `make -C oracle ref`) started from depth-zero PathStates other than
PathState::create_initial, on the cornell_spheres_256 scene (all three closure kinds, power MIS,
depth 16, Russian roulette).

The states cover what the reference's CUDA tests start paths from besides create_initial: zero
throughput (CudaCornellWavefrontSmokeTest TerminatesZeroThroughputBeforeSampling), a high
throughput (CudaTransportParityTest), plus seeded throughputs, already accumulated radiance and
eta scales other than 1, and the initial state itself.

Run from the repository root: python tests/golden/make_state_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "blackframe-renderer_b200"))

from bf200 import abi, runtime, scenes  # noqa: E402
from oracle.bindings import Oracle, Reference  # noqa: E402

WORKLOAD = "cornell_spheres_256"
PATHS = 1024


def state_table(rng, n):
    """beta[4], radiance[4], eta per path."""
    beta = np.ones((n, 4), np.float32)
    radiance = np.zeros((n, 4), np.float32)
    eta = np.ones(n, np.float32)
    kind = np.arange(n) % 5
    beta[kind == 1] = 0.0                                                     # zero throughput
    beta[kind == 2] = np.float32(1e30)                                        # high throughput
    sel = kind == 3
    beta[sel] = rng.uniform(0.0, 4.0, (sel.sum(), 4)).astype(np.float32)
    radiance[sel] = rng.uniform(0.0, 10.0, (sel.sum(), 4)).astype(np.float32)
    eta[sel] = rng.uniform(0.25, 4.0, sel.sum()).astype(np.float32)
    sel = kind == 4
    beta[sel, 1] = 0.0                                                        # one dark lane
    radiance[sel] = np.float32(0.5)
    eta[sel] = np.float32(2.25)
    return beta, radiance, eta


def states_from(beta, radiance, eta):
    n = len(eta)
    states = (abi.PathState * n)()
    for k in range(n):
        for lane in range(4):
            states[k].beta[lane] = float(beta[k, lane])
            states[k].radiance[lane] = float(radiance[k, lane])
        states[k].eta_scale = float(eta[k])
    return states


def inputs_for(samples, width, height):
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    rays = Oracle().camera_rays(cam, samples)
    inputs = (abi.PathInput * len(samples))()
    for k in range(len(samples)):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    return inputs


def sample_table(rng, n, width, height):
    table = np.stack([rng.integers(0, width, n), rng.integers(0, height, n), rng.integers(0, 1 << 40, n),
                      np.full(n, 0x243F6A8885A308D3)], axis=1).astype(np.uint64)
    samples = (abi.SampleIndex * n)()
    for k in range(n):
        samples[k].pixel_x, samples[k].pixel_y = int(table[k, 0]), int(table[k, 1])
        samples[k].sample_index, samples[k].seed = int(table[k, 2]), int(table[k, 3])
    return table, samples


def main():
    rng = np.random.default_rng(20261205)
    builder, options, (width, height, _) = scenes.build_workload(WORKLOAD)
    table, samples = sample_table(rng, PATHS, width, height)
    beta, radiance, eta = state_table(rng, PATHS)
    ref = Reference()
    handle = ref.scene(builder)
    results, failures = ref.trace_states(handle, inputs_for(samples, width, height),
                                         states_from(beta, radiance, eta), options)
    ref.destroy(handle)
    out = {"samples": table, "beta_in": beta, "radiance_in": radiance, "eta_in": eta,
           "radiance": np.array([list(r.radiance) for r in results], np.float32),
           "beta": np.array([list(r.beta) for r in results], np.float32),
           "eta": np.array([r.eta_scale for r in results], np.float32),
           "depth": np.array([r.depth for r in results], np.uint32),
           "termination": np.array([r.termination for r in results], np.uint32),
           "lane_status": np.array([r.lane_status for r in results], np.uint32)}
    np.savez_compressed(os.path.join(HERE, "initial_states.npz"), **out)
    print(f"{PATHS} paths, {failures} refused by the reference, terminations "
          f"{np.bincount(out['termination'], minlength=5).tolist()}")


if __name__ == "__main__":
    main()
