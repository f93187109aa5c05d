"""The environment-map light on the device (bf200_environment_map_*; EnvironmentMapLightT<float> of
EnvironmentLights.hpp) against the oracle and the reference's golden outputs.

* Bit for bit against the oracle with device trig rounding, on every golden case and on fresh
  random maps: samples (direction, radiance, pdf, status), pdf_li, le and power.
* Against the reference's own outputs (tests/golden/envmap.npz): the same statuses, texels, pdfs
  and radiances everywhere; sample directions bit-equal except where the reference's C-library
  sine or cosine of the sampled azimuth is an ulp off the correctly rounded value the device uses
  (a few percent of samples), and then within 1e-6.
* The C ABI's packet binding and malformed-map refusals.
"""
import numpy as np
import pytest

from bf200 import runtime
from bf200.envmap import EnvironmentMap
from oracle.bindings import oracle_environment

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    with runtime.Context(0, path_capacity=1 << 12) as c:
        yield c


@pytest.fixture(scope="module")
def golden():
    import os
    return dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "envmap.npz")))


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8).reshape(len(a), -1)


def compare_with_oracle(device, oracle, canonical, unit, free, bounds):
    got, expected = device.sample(canonical), oracle.sample(canonical)
    assert (bits(got) == bits(expected)).all(), f"{(bits(got) != bits(expected)).any(1).sum()} samples differ"
    for query, dirs in (("pdf", unit), ("le", free)):
        g_value, g_status = getattr(device, query)(dirs)
        e_value, e_status = getattr(oracle, query)(dirs)
        assert (g_status == e_status).all(), query
        assert (g_value.view(np.uint32) == e_value.view(np.uint32)).all(), query
    for lo, hi in bounds:
        rc, power = oracle.power(lo, hi)
        if rc == 0:
            assert (device.power(lo, hi).view(np.uint32) == power.view(np.uint32)).all()
        else:
            with pytest.raises(runtime.Bf200Error):
                device.power(lo, hi)


def test_device_equals_the_oracle_on_the_golden_cases(ctx, golden):
    for name in golden["names"]:
        name = str(name)
        texels, q = golden[f"{name}/texels"], golden[f"{name}/quaternion"]
        with EnvironmentMap(ctx, texels, golden["nanometers"], q) as device:
            oracle = oracle_environment(texels, golden["nanometers"], q, device_trig=True)
            compare_with_oracle(device, oracle, golden[f"{name}/canonical"], golden[f"{name}/pdf_directions"],
                                golden[f"{name}/le_directions"], golden["bounds"])
            oracle.close()


def test_device_equals_the_oracle_on_fresh_maps(ctx):
    rng = np.random.default_rng(2026)
    nm = np.array([390.0, 480.0, 610.0, 790.0], np.float32)
    for _ in range(8):
        h, w = int(rng.integers(1, 40)), int(rng.integers(1, 80))
        texels = rng.gamma(0.5, 2.0, (h, w, 4)).astype(np.float32)
        texels[rng.random((h, w)) < 0.2] = 0.0
        texels[..., 3][rng.random((h, w)) < 0.3] = 0.0
        if not texels.any():
            texels[0, 0] = 1.0
        q = rng.normal(size=4)
        q = (q / np.linalg.norm(q)).astype(np.float32)
        u = rng.random((20000, 2)).astype(np.float32)
        d = rng.normal(size=(5000, 3))
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        with EnvironmentMap(ctx, texels, nm, q) as device:
            oracle = oracle_environment(texels, nm, q, device_trig=True)
            compare_with_oracle(device, oracle, u, d, d * rng.uniform(0.01, 100, (len(d), 1)).astype(np.float32),
                                [([-1, -1, -1], [1, 1, 1]), ([-3, 0, 2], [5, 9, 2.5])])
            oracle.close()


def test_device_against_the_reference_golden_outputs(ctx, golden):
    total = exact = 0
    for name in golden["names"]:
        name = str(name)
        with EnvironmentMap(ctx, golden[f"{name}/texels"], golden["nanometers"], golden[f"{name}/quaternion"]) as m:
            got = m.sample(golden[f"{name}/canonical"])
            ref = golden[f"{name}/sample"]
            assert ((got["status"] == 0) == (ref["status"] == 0)).all()
            assert (got["valid"] == ref["valid"]).all()
            assert (got["pdf"].view(np.uint32) == ref["pdf"].view(np.uint32)).all()
            assert (got["radiance"].view(np.uint32) == ref["radiance"].view(np.uint32)).all()
            assert np.abs(got["direction"] - ref["direction"]).max() <= 1e-6
            exact += int((got["direction"].view(np.uint32) == ref["direction"].view(np.uint32)).all(1).sum())
            total += len(got)
            pdf, status = m.pdf(golden[f"{name}/pdf_directions"])
            assert ((status == 0) == (golden[f"{name}/pdf_status"] == 0)).all()
            same = pdf.view(np.uint32) == golden[f"{name}/pdf"].view(np.uint32)
            assert same.mean() >= 0.99, f"{name}: pdf equal on {same.mean():.4f}"
            le, status = m.le(golden[f"{name}/le_directions"])
            assert ((status == 0) == (golden[f"{name}/le_status"] == 0)).all()
            same = (le.view(np.uint32) == golden[f"{name}/le"].view(np.uint32)).all(1)
            assert same.mean() >= 0.99, f"{name}: le equal on {same.mean():.4f}"
    print(f"sample directions bit-equal to the reference on {exact}/{total}")
    assert exact >= 0.95 * total


def test_packet_binding_and_malformed_maps_are_refused(ctx):
    nm = [400.0, 500.0, 600.0, 700.0]
    with EnvironmentMap(ctx, np.ones((2, 4, 4), np.float32), nm) as m:
        other = EnvironmentMap.__new__(EnvironmentMap)
        other.__dict__.update(m.__dict__)
        other.nanometers = np.array([400.0, 500.0, 600.0, 701.0], np.float32)
        with pytest.raises(runtime.Bf200Error):
            other.sample(np.array([[0.5, 0.5]], np.float32))
        assert len(m.sample(np.zeros((0, 2), np.float32))) == 0
    for texels, q in ((np.full((1, 1, 4), -1.0, np.float32), (0, 0, 0, 1)),
                      (np.ones((1, 1, 4), np.float32), (0, 0, 0, 2)),
                      (np.full((1, 1, 4), np.nan, np.float32), (0, 0, 0, 1))):
        with pytest.raises(runtime.Bf200Error):
            EnvironmentMap(ctx, texels, nm, q)
