"""Freezes golden outputs of the reference's own environment-map light (EnvironmentMapLightT<float>,
EnvironmentLights.hpp) into tests/golden/envmap.npz, through the reference compiled from its tree
(oracle/_ref/libbfref.so, `make -C oracle ref REF=<reference tree>`; entry points in
oracle/ref_envmap.cpp). Run from the repository root: python tests/golden/make_envmap_golden.py

Cases (seeded): maps of several shapes -- random, sparse with zero texels and zero lanes, a smooth
sky with a sun, 2x1 and 1x64 partitions, a constant 1x1, a black map -- under identity and
non-trivial rotations. Per case: sample_li on random canonical pairs plus the edges and CDF
boundaries; pdf_li on random unit directions, the axes and invalid directions; le on directions of
any length, zero and non-finite ones; power over several scene bounds. Creation failures of
malformed inputs are stored with the reference's status code.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "blackframe-renderer_b200"))

from oracle.bindings import CheckerError, reference_environment  # noqa: E402

NANOMETERS = np.array([412.5, 530.0, 647.5, 765.0], np.float32)


def unit_quaternion(v):
    v = np.asarray(v, np.float64)
    return (v / np.linalg.norm(v)).astype(np.float32)


def maps():
    rng = np.random.default_rng(20261204)
    out = {}
    out["random_8x4"] = (rng.uniform(0.0, 2.0, (4, 8, 4)), unit_quaternion([0.1, 0.7, -0.2, 0.5]))
    sparse = rng.uniform(0.0, 5.0, (8, 16, 4))
    sparse[rng.random((8, 16)) < 0.6] = 0.0
    sparse[..., 2][rng.random((8, 16)) < 0.5] = 0.0
    out["sparse_16x8"] = (sparse, np.array([np.sin(np.pi / 4), 0.0, 0.0, np.cos(np.pi / 4)], np.float32))
    theta = (np.arange(32) + 0.5) / 32 * np.pi
    phi = (np.arange(64) + 0.5) / 64 * 2 * np.pi
    sky = np.zeros((32, 64, 4))
    sky += (0.3 + 0.7 * np.clip(np.cos(theta), 0, 1))[:, None, None] * np.array([0.4, 0.6, 0.9, 1.0])
    sky[7, 20] = [4000.0, 3500.0, 3000.0, 2500.0]
    sky += 0.05 * np.cos(phi)[None, :, None] ** 2
    out["sky_64x32"] = (sky, unit_quaternion([0.02, 0.3, 0.01, 0.95]))
    out["contract_2x1"] = (np.array([[[1.0, 2.0, 3.0, 4.0], [0.5, 0.5, 0.5, 0.5]]]), unit_quaternion([0, 0, 0, 1]))
    out["tall_1x64"] = (rng.uniform(0.1, 1.0, (64, 1, 4)), unit_quaternion([0.3, -0.1, 0.4, 0.8]))
    out["constant_1x1"] = (np.full((1, 1, 4), 0.75), unit_quaternion([0, 0, 0, 1]))
    out["black_4x2"] = (np.zeros((2, 4, 4)), unit_quaternion([0, 1, 0, 1]))
    return {k: (np.asarray(t, np.float32), q) for k, (t, q) in out.items()}


def canonical_inputs(rng):
    u = rng.random((1024, 2)).astype(np.float32)
    edges = np.array([[0.0, 0.0], [np.nextafter(np.float32(1), np.float32(0)), 0.0],
                      [0.0, np.nextafter(np.float32(1), np.float32(0))], [0.5, 0.5]], np.float32)
    # the grid of multiples of 1/16, which holds CDF entries of the small tables (a sample equal to an
    # entry selects the next interval)
    cdf_values = np.array([[(i % 16) / 16.0, ((i // 16) % 16) / 16.0] for i in range(256)], np.float32)
    invalid = np.array([[1.0, 0.5], [-0.0, 0.2], [np.nan, 0.1], [0.3, np.inf], [-1e-8, 0.4]], np.float32)
    return np.concatenate([u, edges, cdf_values, invalid])


def direction_inputs(rng, unit):
    d = rng.normal(size=(512, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    if not unit:
        d *= rng.uniform(1e-3, 1e3, (len(d), 1))
    axes = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.float64)
    seam = np.array([[1.0, 0.3, -1e-9], [1.0, -0.2, 1e-9], [0.6, 0.0, 0.8]], np.float64)
    seam /= np.linalg.norm(seam, axis=1, keepdims=True)
    bad = np.array([[0, 0, 0], [np.nan, 0, 1], [np.inf, 0, 0], [2, 0, 0], [1e-30, 0, 0]], np.float64)
    return np.concatenate([d, axes, seam, bad]).astype(np.float32)


BOUNDS = np.array([[[-1, -1, -1], [1, 1, 1]], [[-40, -12, -40], [40, 12, 40]], [[-1, 0, -1], [1, 0, 1]],
                   [[2, 2, 2], [2, 2, 2]], [[-1e30, -1e30, -1e30], [1e30, 1e30, 1e30]],
                   [[1, 0, 0], [-1, 1, 1]]], np.float32)

INVALID = {
    "zero_width": (np.zeros((1, 0, 4), np.float32), [0, 0, 0, 1], NANOMETERS),
    "negative_texel": (np.array([[[1, -1, 1, 1]]], np.float32), [0, 0, 0, 1], NANOMETERS),
    "nan_texel": (np.array([[[1, np.nan, 1, 1]]], np.float32), [0, 0, 0, 1], NANOMETERS),
    "not_unit_rotation": (np.ones((1, 2, 4), np.float32), [0, 0, 0, 1.001], NANOMETERS),
    "invisible_wavelength": (np.ones((1, 2, 4), np.float32), [0, 0, 0, 1], [300.0, 500.0, 600.0, 700.0]),
}


def main():
    rng = np.random.default_rng(7)
    arrays = {"nanometers": NANOMETERS, "bounds": BOUNDS}
    names = []
    for name, (texels, q) in maps().items():
        light = reference_environment(texels, NANOMETERS, q)
        u = canonical_inputs(rng)
        unit = direction_inputs(rng, True)
        free = direction_inputs(rng, False)
        s = light.sample(u)
        pdf, pdf_status = light.pdf(unit)
        le, le_status = light.le(free)
        powers = [light.power(lo, hi) for lo, hi in BOUNDS]
        arrays.update({
            f"{name}/texels": texels, f"{name}/quaternion": q, f"{name}/canonical": u, f"{name}/sample": s,
            f"{name}/pdf_directions": unit, f"{name}/pdf": pdf, f"{name}/pdf_status": pdf_status,
            f"{name}/le_directions": free, f"{name}/le": le, f"{name}/le_status": le_status,
            f"{name}/power_status": np.array([p[0] for p in powers], np.int32),
            f"{name}/power": np.stack([p[1] for p in powers]),
        })
        light.close()
        names.append(name)
        print(name, "samples", int(s["valid"].sum()), "failed", int((s["status"] != 0).sum()))
    codes = []
    for name, (texels, q, nm) in INVALID.items():
        try:
            reference_environment(texels, nm, q).close()
            codes.append(0)
        except CheckerError as e:
            codes.append(int(str(e).split(":")[0]))
        print(name, codes[-1])
    arrays["invalid_names"] = np.array(list(INVALID))
    arrays["invalid_codes"] = np.array(codes, np.int32)
    arrays["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "envmap.npz"), **arrays)


if __name__ == "__main__":
    main()
