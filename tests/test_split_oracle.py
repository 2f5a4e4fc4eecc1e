"""CPU checks of the split-precision oracle (int8 slices, exact int32 sums)."""
from __future__ import annotations

import numpy as np

from oracle import split as S


def _rand(shape, rng):
    return rng.normal(size=shape) + 1j * rng.normal(size=shape)


def test_slices_reconstruct_the_lines():
    rng = np.random.default_rng(0)
    X = rng.normal(size=(7, 33)) * np.logspace(-3, 3, 33)[None, :]
    for s in (2, 4, 8):
        sl, e = S.slice_lines(X, s)
        assert np.all(np.abs(sl.astype(int)) <= 127)
        back = sum(np.ldexp(sl[i].astype(float), -7 * (i + 1)) for i in range(s))
        back = np.ldexp(back, e[:, None])
        err = np.max(np.abs(back - X), axis=1) / np.max(np.abs(X), axis=1)
        assert np.all(err < 2.0 ** (-7 * s + 1))


def test_zero_lines_and_exact_powers_of_two():
    X = np.zeros((3, 5))
    X[1, 2] = 1.0                     # max exactly 2^0 -> e = 1, slice 64
    X[2, 0] = -0.75
    sl, e = S.slice_lines(X, 3)
    assert list(e) == [0, 1, 0]
    assert sl[0, 1, 2] == 64 and np.all(sl[1:, 1, 2] == 0)
    assert sl[0, 2, 0] == -96


def test_ozaki_error_falls_two_decades_per_slice():
    rng = np.random.default_rng(1)
    A = _rand((40, 60), rng)
    B = _rand((60, 30), rng)
    C = A @ B
    errs = [np.max(np.abs(S.ozaki_zgemm(A, B, s) - C)) / np.max(np.abs(C)) for s in range(2, 9)]
    for a, b in zip(errs[:-1], errs[1:]):
        assert b < a / 30.0
    assert errs[-1] < 1e-14


def test_real_forms_give_the_complex_product():
    rng = np.random.default_rng(2)
    A = _rand((5, 4), rng)
    B = _rand((4, 3), rng)
    Ap, Bt = S.real_forms(A, B)
    Cp = Ap @ Bt.T
    np.testing.assert_allclose(Cp[:, 0::2] + 1j * Cp[:, 1::2], A @ B, rtol=1e-14, atol=1e-14)
