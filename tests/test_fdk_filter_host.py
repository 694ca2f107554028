"""The FDK ramp filter's host side (ct2b200.fdk_filter), without a GPU: the
2n-1 convolution taps reproduce the reference's filtering of a detector line
-- zero-pad to npad = 2^round(log2(2n-1)), multiply the FFT by the frequency
response, keep the first n samples of the real inverse FFT
(emil_code/FDK.py:33-79) -- for plain and Hann-windowed ramps, and the
frequency grid follows setFreqrange.kappa1D."""
import numpy as np
import pytest

from ct2b200 import fdk_filter as F


def _reference_filtering(line, dp, opt_window, L):
    n = line.shape[-1]
    npad, filt = F.frequency_response(dp, n, opt_window, L)
    padded = np.zeros(line.shape[:-1] + (npad,))
    padded[..., :n] = line
    return np.real(np.fft.ifft(filt * np.fft.fft(padded)))[..., :n]


def _tap_filtering(line, dp, opt_window, L):
    n = line.shape[-1]
    taps = F.convolution_taps(dp, n, opt_window, L).astype(np.float64)
    # out[i] = sum_j line[j] * h[i - j], taps[k] = h[k - (n - 1)]
    return np.stack([np.convolve(row, taps)[n - 1:2 * n - 1] for row in line.reshape(-1, n)])


@pytest.mark.parametrize("n", [5, 16, 33, 100])
@pytest.mark.parametrize("dp", [0.5, 1.3])
@pytest.mark.parametrize("opt_window, L", [("", 1), ("Hann", 1), ("Hann", 0.7)])
def test_taps_equal_the_padded_fft_filtering(n, dp, opt_window, L):
    rng = np.random.default_rng(n)
    lines = rng.random((3, n))
    want = _reference_filtering(lines, dp, opt_window, L)
    got = _tap_filtering(lines, dp, opt_window, L)
    # the taps are stored in FP32
    assert np.max(np.abs(got - want)) <= 1e-6 * np.max(np.abs(want))


def test_padding_length_and_tap_count():
    for n, npad in ((5, 8), (16, 32), (33, 64), (100, 256), (384, 1024)):
        assert F.frequency_response(1.0, n)[0] == npad
        taps = F.convolution_taps(1.0, n)
        assert taps.shape == (2 * n - 1,) and taps.dtype == np.float32
        assert not taps.flags.writeable
    # the ramp is even: lag k and lag -k carry the same tap
    taps = F.convolution_taps(0.8, 40, "Hann", 1)
    assert np.array_equal(taps, taps[::-1])


def test_kappa1d_grid():
    assert np.allclose(F.kappa1D(4, 0.5), np.array([-2, -1, 0, 1]) / 2.0)
    assert np.allclose(F.kappa1D(5, 2.0), np.array([-2, -1, 0, 1, 2]) / 10.0)
