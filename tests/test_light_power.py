"""Power-weighted light selection (bf200_light_power_cdf, the CDF bf200_scene_set_light_powers
installs) against the reference's LightSampler::create_power_weighted: every light's selection
probability and the selection of random canonical samples, bit for bit, on seeded power sets
(zero-power lights, lanes of very different scales, one light), plus the refusals. The reference
values come from the compiled reference where it exists, else from tests/golden/light_power.npz
(made by tests/golden/make_light_power_golden.py). Host code only."""
import os

import numpy as np
import pytest

from bf200 import runtime

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "light_power.npz")


def select(cdf, u):
    """LightSampler::sample on the boundaries: upper_bound over boundaries[1:], probability = width;
    a sample at or beyond the last boundary (u = 1 after rounding to float) selects nothing, and
    the reference reports an error for it (index 0xFFFFFFFF, probability -1 in the fixture)."""
    index = int(np.searchsorted(cdf[1:], np.float32(u), side="right"))
    if index >= len(cdf) - 1:
        return 0xFFFFFFFF, np.float32(-1.0)
    return index, np.float32(cdf[index + 1] - cdf[index])


def test_power_cdf_matches_the_reference():
    g = np.load(GOLDEN)
    for k in range(int(g["sets"])):
        powers, samples = g[f"powers_{k}"], g[f"samples_{k}"]
        cdf = runtime.light_power_cdf(powers)
        probabilities = (cdf[1:] - cdf[:-1]).astype(np.float32)
        assert np.array_equal(probabilities.view(np.uint32), g[f"probabilities_{k}"].view(np.uint32)), k
        for j, u in enumerate(samples):
            index, p = select(cdf, u)
            assert index == g[f"selected_{k}"][j] and p.view(np.uint32) == g[f"selected_probability_{k}"][j].view(
                np.uint32), (k, j)


def test_power_cdf_refusals():
    for powers in ([[0, 0, 0, 0]], [[1, -1, 0, 0]], [[1, np.inf, 0, 0]], [[np.nan, 0, 0, 0]]):
        with pytest.raises(runtime.Bf200Error):
            runtime.light_power_cdf(np.array(powers, np.float32))


def test_oracle_power_weighted_transport_matches_the_compiled_reference():
    """The oracle's power-weighted selection inside transport against the reference's own
    trace_scene_mis with LightSampler::create_power_weighted (512 paths of a three-light box).
    Runs where the reference was compiled (oracle/_ref)."""
    from oracle.bindings import Oracle, Reference, reference_available
    if not reference_available():
        pytest.skip("oracle/_ref not built here")
    from bf200 import abi
    from helpers import REFERENCE_DIVERGED_FRACTION, arrays, check_paths
    from test_gpu_light_power import light_powers, path_inputs, three_light_box
    builder = three_light_box()
    powers = light_powers(builder)
    oracle, ref = Oracle(), Reference()
    inputs = path_inputs(oracle, 512, 21)
    options = abi.default_options(mis="power", max_depth=8)
    h = oracle.scene(builder)
    oracle.set_light_powers(h, powers)
    got, failures = oracle.trace(h, inputs, options)
    oracle.destroy(h)
    h = ref.scene(builder)
    ref.set_light_powers(h, powers)
    want, ref_failures = ref.trace(h, inputs, options)
    ref.destroy(h)
    assert failures == 0 and ref_failures == 0
    exact, _ = check_paths(arrays(got), arrays(want), "oracle vs reference, power-weighted",
                           diverged=REFERENCE_DIVERGED_FRACTION)
    assert exact >= 0.99
