"""Sobol and Owen-scrambled Sobol bits: the library functions (bf200_sobol_bits,
bf200_owen_sobol_bits) and the oracle's restatement against the reference's known answers, and
against the compiled reference on random inputs where it is built.

Known answers: the first ten points of the first three dimensions published with the Joe-Kuo
directions and the full-table, full-index-width bits of Tests/Renderer/SobolSamplingTest.cpp:
29-58; the frozen nested-scramble words of Tests/Renderer/OwenScramblingTest.cpp:29-81.
"""
import numpy as np
import pytest

from bf200 import runtime
from oracle.bindings import Oracle, Reference, reference_available

U64 = (1 << 64) - 1
FIRST_TEN = [(0, 0, 0), (8, 8, 8), (12, 4, 4), (4, 12, 12), (6, 6, 10), (14, 14, 2), (10, 2, 14), (2, 10, 6),
             (3, 5, 15), (11, 13, 7)]
SOBOL_KNOWN = [
    (0x0123456789ABCDEF, 63, 0x013E8C6349603C80),
    (0x0123456789ABCDEF, 255, 0xB321991D6689DC80),
    (0x0123456789ABCDEF, 1023, 0xE4BCA0B1ED509A80),
    (0x0123456789ABCDEF, 4095, 0x572DD6D8275D9480),
    (0x0123456789ABCDEF, 16383, 0x66A5274EF5FA7480),
    (0x0123456789ABCDEF, 21200, 0xF4C1FC94854F3780),
    (0x8000000000000000, 21200, 0x45AC83CC9F734085),
    (U64, 21200, 0xA8D3F37AB495C0C3),
    (U64, 1, U64),
]
# (pixel_x, pixel_y, sample_index, seed, dimension, bits)
OWEN_KNOWN = [
    (0, 0, 0, 0, 0, 0x92A8B3FFD11450D8),
    (0, 0, 1, 0, 0, 0x05425D9FC8F958EF),
    (0, 0, 2, 0x0123456789ABCDEF, 0, 0x2D5F4AEE875D131D),
    (0, 0, 0x0123456789ABCDEF, 0x0123456789ABCDEF, 63, 0x952C2015E62C23E3),
    (113, 47, 0x0123456789ABCDEF, 0xA5A5F00D12345678, 63, 0xA694114D8B9547EF),
    (0, 0, 0x0123456789ABCDEF, 0xFEDCBA9876543210, 255, 0x210EA3A92DEE7EFC),
    (0, 0, 0x0123456789ABCDEF, 0, 21200, 0x8A185723D91F9C0B),
    (0, 0, 0x8000000000000000, U64, 21200, 0x5E46341BD2FA3170),
    (0, 0, U64, 0x0123456789ABCDEF, 21200, 0x3731AD8327D19D7C),
]


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


def test_first_ten_published_points():
    for sample, numerators in enumerate(FIRST_TEN):
        for dim, numerator in enumerate(numerators):
            assert runtime.sobol_bits(sample, dim) == numerator << 60


def test_sobol_known_answers(oracle):
    for sample, dim, bits in SOBOL_KNOWN:
        assert runtime.sobol_bits(sample, dim) == bits
        assert oracle.sobol_bits(sample, dim) == bits


def test_owen_frozen_vectors(oracle):
    for px, py, sample, seed, dim, bits in OWEN_KNOWN:
        assert runtime.owen_sobol_bits(px, py, sample, seed, dim) == bits
        assert oracle.owen_sobol_bits(px, py, sample, seed, dim) == bits


def test_dimensions_outside_the_table_are_refused():
    for dim in (21201, U64):
        with pytest.raises(runtime.Bf200Error) as info:
            runtime.sobol_bits(37, dim)
        assert info.value.status == 5
        with pytest.raises(runtime.Bf200Error):
            runtime.owen_sobol_bits(0, 0, 37, 0, dim)


def test_dyadic_stratification_of_scrambled_points():
    # every 2^k prefix of a scrambled Sobol dimension covers each of the 2^k bins once
    for dim in (0, 5, 63, 1023):
        values = [runtime.owen_sobol_bits(7, 9, i, 0x1234, dim) >> 52 for i in range(4096)]
        assert sorted(values) == list(range(4096))


@pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built (reference tree absent)")
def test_random_inputs_match_the_compiled_reference(oracle):
    ref = Reference()
    rng = np.random.default_rng(17)
    for _ in range(400):
        dim = int(rng.integers(0, 21201))
        sample = int(rng.integers(0, 1 << 63)) * 2 + int(rng.integers(0, 2))
        px, py = int(rng.integers(0, 1 << 32)), int(rng.integers(0, 1 << 32))
        seed = int(rng.integers(0, 1 << 63)) * 2 + int(rng.integers(0, 2))
        expected = ref.sobol_bits(sample, dim)
        assert runtime.sobol_bits(sample, dim) == expected
        assert oracle.sobol_bits(sample, dim) == expected
        expected = ref.owen_sobol_bits(px, py, sample, seed, dim)
        assert runtime.owen_sobol_bits(px, py, sample, seed, dim) == expected
        assert oracle.owen_sobol_bits(px, py, sample, seed, dim) == expected
