"""Writes tests/golden/light_power.npz: the reference's power-weighted LightSampler
(LightSampler::create_power_weighted, compiled into oracle/_ref/libbfref.so by `make -C oracle ref`)
on seeded 4-lane power sets: every light's selection probability and the selection of 64 seeded
canonical samples. Run from the repository root: python tests/golden/make_light_power_golden.py"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "blackframe-renderer_b200"))

from oracle.bindings import Reference  # noqa: E402


def power_sets(rng):
    sets = [np.array([[1.0, 1.0, 1.0, 1.0]], np.float32),                          # one light
            np.array([[17, 17, 17, 17], [0, 0, 0, 0], [3, 5, 7, 11]], np.float32),   # a zero-power light
            np.array([[0, 0, 0, 0], [2, 0, 0, 0], [0, 0, 0, 0]], np.float32)]        # zero lights at both ends
    for n in (2, 5, 17, 200, 2048):
        p = rng.lognormal(0.0, 2.0, (n, 4)).astype(np.float32)
        p[rng.random((n, 4)) < 0.1] = 0.0
        sets.append(p)
    sets.append((rng.random((64, 4)) * np.float32(1e-30)).astype(np.float32))      # tiny powers
    sets.append((rng.random((64, 4)) * np.float32(1e30)).astype(np.float32))       # huge powers
    return sets


def main():
    ref = Reference()
    rng = np.random.default_rng(20261203)
    out = {}
    for k, powers in enumerate(power_sets(rng)):
        samples = np.concatenate([rng.random(60), [0.0, 0.5, np.nextafter(1.0, 0.0), 1e-9]]).astype(np.float32)
        result, code = ref.power_sampler(powers, samples)
        assert code == 0, (k, code)
        probabilities, selected, selected_probability = result
        out.update({f"powers_{k}": powers, f"samples_{k}": samples, f"probabilities_{k}": probabilities,
                    f"selected_{k}": selected, f"selected_probability_{k}": selected_probability})
    out["sets"] = np.int64(len(power_sets(np.random.default_rng(20261203))))
    np.savez_compressed(os.path.join(HERE, "light_power.npz"), **out)
    print("sets:", out["sets"])


if __name__ == "__main__":
    main()
