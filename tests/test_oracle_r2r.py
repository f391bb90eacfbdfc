"""Pins the oracle's r2r transforms to FFTW's published definitions.

scipy.fft.dct/dst with norm=None, types 2 and 3, are defined exactly as FFTW's REDFT10,
REDFT01, RODFT10 and RODFT01 (the kinds the reference plans, e.g.
no-adv/cosNoAdvTrackSing.cpp:342-375 and adv/cosAdvTrackMult.cpp:419-467).
"""
import numpy as np
import pytest
import scipy.fft as sf

import oracle

REF = {
    oracle.REDFT10: lambda x, ax=-1: sf.dct(x, 2, axis=ax),
    oracle.REDFT01: lambda x, ax=-1: sf.dct(x, 3, axis=ax),
    oracle.RODFT10: lambda x, ax=-1: sf.dst(x, 2, axis=ax),
    oracle.RODFT01: lambda x, ax=-1: sf.dst(x, 3, axis=ax),
}


@pytest.mark.parametrize("n", [2, 3, 4, 5, 6, 8, 12, 15, 16, 20, 24, 30, 32, 48, 64, 96, 100, 128, 160, 256])
@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_r2r_1d_matches_fftw_definitions(n, kind):
    x = np.random.default_rng(n * 7 + kind).standard_normal(n)
    ref = REF[kind](x)
    got = oracle.r2r_1d(x, kind)
    assert np.max(np.abs(got - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))


KINDS3 = [(0, 0, 0), (1, 1, 1), (2, 0, 0), (0, 2, 0), (0, 0, 2), (3, 1, 1), (1, 3, 1), (1, 1, 3)]


@pytest.mark.parametrize("kinds", KINDS3)
def test_r2r_3d_separable(kinds):
    x = np.random.default_rng(11).standard_normal((6, 10, 8))
    ref = x
    for ax, k in enumerate(kinds):
        ref = REF[k](ref, ax)
    got = oracle.r2r_3d(x, kinds)
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_inverse_pairs_scale_2n():
    # REDFT01(REDFT10(x)) = 2n x and RODFT01(RODFT10(x)) = 2n x (FFTW's normalisation)
    x = np.random.default_rng(3).standard_normal(24)
    for f, b in [(0, 1), (2, 3)]:
        y = oracle.r2r_1d(oracle.r2r_1d(x, f), b)
        assert np.allclose(y, 2 * 24 * x, rtol=0, atol=1e-12)
