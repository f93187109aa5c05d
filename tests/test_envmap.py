"""The environment-map light on the CPU: the oracle's restatement (oracle/bfo_envmap.cpp) and the
product's table construction it links (csrc/bf200_envmap.cpp) against the reference's own
EnvironmentMapLightT<float> (EnvironmentLights.hpp).

* Golden outputs of the compiled reference (tests/golden/envmap.npz, made by
  tests/golden/make_envmap_golden.py): sample_li, pdf_li, le and power equal bit for bit, with the
  C library's float trig that the reference calls, and the same creation failures.
* Where oracle/_ref is built here, the same comparison on fresh random maps and rotations.
* The reference's own test properties (Tests/Renderer/Light/EnvironmentLightsTest.cpp): the pdf of
  a sample is the pdf_li of its direction and le of that direction its radiance; the solid-angle
  pdf integrates to one; texels are chosen in proportion to mean radiance times solid angle; a
  constant map is uniform; power does not depend on the rotation; black maps give no samples.
"""
import numpy as np
import pytest

from oracle.bindings import CheckerError, oracle_environment, reference_available, reference_environment

GOLDEN = None


def golden():
    global GOLDEN
    if GOLDEN is None:
        import os
        GOLDEN = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "envmap.npz")))
    return GOLDEN


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8).reshape(len(a), -1) if a.ndim else a.view(np.uint8)


def case_names():
    return [str(n) for n in golden()["names"]]


@pytest.mark.parametrize("name", case_names())
def test_oracle_equals_the_reference_golden_outputs(name):
    g = golden()
    light = oracle_environment(g[f"{name}/texels"], g["nanometers"], g[f"{name}/quaternion"])
    got = light.sample(g[f"{name}/canonical"])
    expected = g[f"{name}/sample"]
    assert (bits(got) == bits(expected)).all(), f"{(bits(got) != bits(expected)).any(1).sum()} samples differ"
    pdf, status = light.pdf(g[f"{name}/pdf_directions"])
    assert (pdf.view(np.uint32) == g[f"{name}/pdf"].view(np.uint32)).all()
    assert ((status == 0) == (g[f"{name}/pdf_status"] == 0)).all()
    le, le_status = light.le(g[f"{name}/le_directions"])
    assert (le.view(np.uint32) == g[f"{name}/le"].view(np.uint32)).all()
    assert ((le_status == 0) == (g[f"{name}/le_status"] == 0)).all()
    for k, (lo, hi) in enumerate(g["bounds"]):
        rc, power = light.power(lo, hi)
        assert (rc == 0) == (g[f"{name}/power_status"][k] == 0)
        assert (power.view(np.uint32) == g[f"{name}/power"][k].view(np.uint32)).all()
    light.close()


def test_malformed_maps_fail_as_in_the_reference():
    g = golden()
    inputs = {
        "zero_width": (np.zeros((1, 0, 4), np.float32), [0, 0, 0, 1], g["nanometers"]),
        "negative_texel": (np.array([[[1, -1, 1, 1]]], np.float32), [0, 0, 0, 1], g["nanometers"]),
        "nan_texel": (np.array([[[1, np.nan, 1, 1]]], np.float32), [0, 0, 0, 1], g["nanometers"]),
        "not_unit_rotation": (np.ones((1, 2, 4), np.float32), [0, 0, 0, 1.001], g["nanometers"]),
        "invisible_wavelength": (np.ones((1, 2, 4), np.float32), [0, 0, 0, 1], [300.0, 500.0, 600.0, 700.0]),
    }
    for name, code in zip(g["invalid_names"], g["invalid_codes"]):
        texels, q, nm = inputs[str(name)]
        with pytest.raises(CheckerError) as failure:
            oracle_environment(texels, nm, q)
        assert int(str(failure.value).split(":")[0]) == code


@pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")
def test_oracle_equals_the_compiled_reference_on_fresh_maps():
    rng = np.random.default_rng(99)
    nm = np.array([380.0, 505.0, 620.0, 801.0], np.float32)
    for trial in range(6):
        h, w = int(rng.integers(1, 24)), int(rng.integers(1, 48))
        texels = rng.exponential(1.0, (h, w, 4)).astype(np.float32)
        texels[rng.random((h, w)) < 0.3] = 0.0
        if not texels.any():
            texels[0, 0, 0] = 1.0
        q = rng.normal(size=4)
        q = (q / np.linalg.norm(q)).astype(np.float32)
        ours, theirs = oracle_environment(texels, nm, q), reference_environment(texels, nm, q)
        u = rng.random((2000, 2)).astype(np.float32)
        assert (bits(ours.sample(u)) == bits(theirs.sample(u))).all()
        d = rng.normal(size=(2000, 3))
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        assert (ours.pdf(d)[0].view(np.uint32) == theirs.pdf(d)[0].view(np.uint32)).all()
        assert (ours.le(d * 7)[0].view(np.uint32) == theirs.le(d * 7)[0].view(np.uint32)).all()
        ours.close()
        theirs.close()


def solid_angles(h, w):
    theta = np.arange(h + 1) * (np.pi / h)
    cos = np.cos(theta)
    return (cos[:-1] - cos[1:])[:, None] * np.full((1, w), 2 * np.pi / w)


def test_sample_pdf_and_emission_agree_with_the_lookups():
    g = golden()
    light = oracle_environment(g["sky_64x32/texels"], g["nanometers"], g["sky_64x32/quaternion"])
    s = light.sample(np.random.default_rng(3).random((4000, 2)).astype(np.float32))
    ok = s["valid"] == 1
    assert ok.all()
    pdf, status = light.pdf(s["direction"])
    assert (status == 0).all() and (pdf == s["pdf"]).all()
    le, status = light.le(s["direction"])
    assert (status == 0).all() and (le == s["radiance"]).all()
    light.close()


def test_pdf_integrates_to_one_and_texels_follow_their_importance():
    rng = np.random.default_rng(5)
    h, w = 8, 16
    texels = rng.uniform(0.1, 3.0, (h, w, 4)).astype(np.float32)
    nm = [400.0, 500.0, 600.0, 700.0]
    light = oracle_environment(texels, nm)
    # the density of a texel is constant over it: probe each texel at its centre direction
    theta = (np.arange(h) + 0.5) * np.pi / h
    phi = (np.arange(w) + 0.5) * 2 * np.pi / w
    dirs = np.stack(np.broadcast_arrays(np.sin(theta)[:, None] * np.cos(phi)[None, :], np.cos(theta)[:, None],
                                        np.sin(theta)[:, None] * np.sin(phi)[None, :]), -1).reshape(-1, 3)
    pdf, status = light.pdf(dirs.astype(np.float32))
    assert (status == 0).all()
    omega = solid_angles(h, w).reshape(-1)
    assert abs(float((pdf.astype(np.float64) * omega).sum()) - 1.0) < 5e-5
    importance = texels.astype(np.float64).sum(-1).reshape(-1) * omega
    expected = importance / importance.sum()
    assert np.allclose(pdf * omega, expected, rtol=2e-5)
    n = 200000
    s = light.sample(rng.random((n, 2)).astype(np.float32))
    counts = np.zeros(h * w)
    _, texel_status = light.pdf(s["direction"])
    assert (texel_status == 0).all()
    # recover the sampled texel from the direction (identity rotation)
    d = s["direction"].astype(np.float64)
    col = np.floor((np.arctan2(d[:, 2], d[:, 0]) % (2 * np.pi)) / (2 * np.pi / w)).astype(int).clip(0, w - 1)
    row = np.floor(np.arccos(np.clip(d[:, 1], -1, 1)) / (np.pi / h)).astype(int).clip(0, h - 1)
    np.add.at(counts, row * w + col, 1)
    sigma = np.sqrt(n * expected * (1 - expected))
    assert (np.abs(counts - n * expected) < 5 * sigma + 2).all()
    light.close()


def test_constant_map_is_uniform_and_power_ignores_rotation():
    nm = [410.0, 520.0, 630.0, 740.0]
    flat = np.full((6, 12, 4), 0.5, np.float32)
    light = oracle_environment(flat, nm)
    d = np.random.default_rng(1).normal(size=(1000, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    pdf, status = light.pdf(d)
    assert (status == 0).all()
    assert np.allclose(pdf, 1.0 / (4.0 * np.pi), rtol=2e-5)
    rc, power = light.power([-1, -1, -1], [1, 1, 1])
    assert rc == 0
    # L * 4 pi * pi r^2 with r = sqrt(3): 0.5 * 4 pi * pi * 3
    assert np.allclose(power, 0.5 * 4 * np.pi * np.pi * 3.0, rtol=1e-5)
    q = np.array([0.3, -0.4, 0.5, 0.7], np.float64)
    rotated = oracle_environment(flat, nm, (q / np.linalg.norm(q)).astype(np.float32))
    assert (rotated.power([-1, -1, -1], [1, 1, 1])[1] == power).all()
    light.close()
    rotated.close()


def test_black_maps_give_no_samples_zero_pdf_and_zero_power():
    light = oracle_environment(np.zeros((2, 3, 4), np.float32), [400.0, 500.0, 600.0, 700.0])
    s = light.sample(np.array([[0.2, 0.7], [0.9, 0.1]], np.float32))
    assert (s["valid"] == 0).all() and (s["status"] == 0).all()
    pdf, status = light.pdf(np.array([[0, 1, 0]], np.float32))
    assert pdf[0] == 0.0 and status[0] == 0
    assert (light.power([-1, -1, -1], [1, 1, 1])[1] == 0).all()
    light.close()
