"""The oracle's textbook mixed-radix FFT against numpy (lengths 2^a 3^b)."""
import numpy as np
import pytest


@pytest.mark.parametrize("n", [1, 2, 3, 4, 6, 8, 12, 16, 18, 24, 27, 32, 48, 64, 96, 128, 192, 384, 1024])
def test_fft_matches_numpy(n):
    import oracle_py as op

    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert np.allclose(op.fft(x, -1), np.fft.fft(x), rtol=0, atol=1e-12 * max(1, n))
    assert np.allclose(op.fft(x, +1), np.fft.ifft(x) * n, rtol=0, atol=1e-12 * max(1, n))


def test_fft_rejects_other_radices():
    import oracle_py as op

    with pytest.raises(ValueError):
        op.fft(np.ones(10, dtype=complex))


def test_mt64_known_answer():
    # std::mt19937_64 default seed 5489: the 10000th draw is 9981545732273789042 (C++ standard).
    import oracle_py as op

    assert int(op.mt64(5489, 10000)[-1]) == 9981545732273789042
