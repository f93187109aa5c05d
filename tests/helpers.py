"""Shared helpers of the test suite: golden inputs as C records, result comparison."""
import numpy as np

from bf200 import abi, scenes

# Per-path radiance tolerance of the parity tests, and the share of paths allowed outside it.
# Against the oracle in its device-rounding mode (Oracle(device_trig=True)) no path may diverge.
# Against outputs of the reference itself, which takes sampled-angle sines and cosines from glibc's
# sinf/cosf (within 0.56 ulp, off the correctly rounded value for about 1.3 % of arguments), a path
# that draws such an angle continues one ulp apart: up to 1 % of paths may then differ.
RELATIVE_TOLERANCE = 1e-5
DIVERGED_FRACTION = 0.0
REFERENCE_DIVERGED_FRACTION = 0.01


def golden_inputs(g):
    n = len(g["pixel_x"])
    inputs = (abi.PathInput * n)()
    for k in range(n):
        r = inputs[k].primary_ray
        for a in range(3):
            r.origin[a] = float(g["ray_origin"][k, a])
            r.direction[a] = float(g["ray_direction"][k, a])
        r.t_min, r.t_max, r.time = 0.0, float("inf"), scenes.PATH_TIME
        r.mask, r.medium = 0xFFFFFFFF, 0
        inputs[k].sample.pixel_x = int(g["pixel_x"][k])
        inputs[k].sample.pixel_y = int(g["pixel_y"][k])
        inputs[k].sample.sample_index = int(g["sample_index"][k])
        inputs[k].sample.seed = 0
    return inputs


def arrays(results):
    n = len(results)
    return {
        "radiance": np.array([list(r.radiance) for r in results], np.float32).reshape(n, 4),
        "beta": np.array([list(r.beta) for r in results], np.float32).reshape(n, 4),
        "depth": np.array([r.depth for r in results], np.uint32),
        "termination": np.array([r.termination for r in results], np.uint32),
        "lane_status": np.array([r.lane_status for r in results], np.uint32),
        "eta": np.array([r.eta_scale for r in results], np.float32),
    }


def bit_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.view(np.uint32) == b.view(np.uint32)


def relative_error(a, b, floor=1e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), floor)


def sensor_from_golden(g):
    s = abi.Sensor()
    for lane in range(4):
        for k in range(3):
            s.response_xyz[lane][k] = float(g["sensor_response"][lane, k])
        s.wavelength_pdf[lane] = float(g["sensor_pdf"][lane])
    s.normalization = float(g["sensor_normalization"])
    return s


def check_paths(got, expected, label, diverged=DIVERGED_FRACTION):
    """Asserts per-path parity (see RELATIVE_TOLERANCE): at most `diverged` of the paths outside
    the tolerance or with another termination; returns the bit-exact and close shares."""
    same = bit_equal(got["radiance"], expected["radiance"]).all(axis=1)
    close = (relative_error(got["radiance"], expected["radiance"]) <= RELATIVE_TOLERANCE).all(axis=1)
    term = got["termination"] == expected["termination"]
    n = len(same)
    print(f"{label}: {same.sum()}/{n} bit-exact, {close.sum()}/{n} within {RELATIVE_TOLERANCE}, "
          f"{term.sum()}/{n} same termination")
    assert (got["lane_status"] == 0).all(), f"{label}: failed lanes {np.nonzero(got['lane_status'])[0][:10]}"
    assert close.mean() >= 1.0 - diverged, f"{label}: only {close.sum()}/{n} within tolerance"
    assert term.mean() >= 1.0 - diverged, f"{label}: terminations differ on {n - term.sum()}/{n}"
    return same.mean(), close.mean()
