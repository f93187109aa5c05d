"""The spatial light tree traversed on the device (bf200_light_tree_select_device) against the
reference's LightSampler::create_spatial_tree selections (tests/golden/light_tree.npz, made by
tests/golden/make_light_tree_golden.py from the compiled reference). The device rounds double
logarithms and exponentials to float where the reference calls the C library's float functions,
so probabilities agree to a relative 1e-5 and selections agree except where a sample lies within
that difference of a branch boundary."""
import numpy as np
import pytest

from bf200 import runtime

pytestmark = pytest.mark.gpu


def test_device_light_tree_matches_the_reference(golden):
    import torch
    g = golden("light_tree")
    total = agree = exact = 0
    for k in range(int(g["sets"])):
        lo, hi, p = g[f"lo_{k}"], g[f"hi_{k}"], g[f"powers_{k}"]
        positions = np.ascontiguousarray(g[f"positions_{k}"], np.float32)
        samples = np.ascontiguousarray(g[f"samples_{k}"], np.float32)
        n = len(samples)
        d_positions = torch.from_numpy(positions.reshape(-1)).cuda()
        d_samples = torch.from_numpy(samples).cuda()
        d_lights = torch.zeros(n, dtype=torch.int32, device="cuda")
        d_probabilities = torch.zeros(n, dtype=torch.float32, device="cuda")
        runtime.light_tree_select_device(lo, hi, p, d_positions.data_ptr(), d_samples.data_ptr(), n,
                                         d_lights.data_ptr(), d_probabilities.data_ptr())
        torch.cuda.synchronize()
        lights = d_lights.cpu().numpy().view(np.uint32)
        probabilities = d_probabilities.cpu().numpy()
        want_lights, want_probabilities = g[f"selected_{k}"], g[f"probability_{k}"]
        same = lights == want_lights
        valid = same & (want_lights != 0xFFFFFFFF)
        relative = np.abs(probabilities.astype(np.float64) - want_probabilities) / np.maximum(
            np.abs(want_probabilities.astype(np.float64)), 1e-30)
        assert (relative[valid] <= 1e-5).all(), (k, float(relative[valid].max()))
        total += n
        agree += int(same.sum())
        exact += int((valid & (probabilities.view(np.uint32) == want_probabilities.view(np.uint32))).sum())
    assert agree >= 0.99 * total, (agree, total)
    print(f"light tree on the device: {agree}/{total} selections agree, {exact} probabilities bit-exact")
