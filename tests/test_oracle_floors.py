"""The FP64 floors that the GPU parity tolerances rest on, measured on the oracle alone (CPU).

Two FP64 floors sit above 1e-12 and come from the reference's own arithmetic,
not from the GPU:
- the carrier-shift methods depend on the last bits of the spectral centroid
  (they decide how the propagation phase of the shifted bins, ~1e4 rad, rounds),
  and the reference sums the centroid in sequence
  (optics/propagate.go:391-416);
- the reference's Bluestein transform forms its chirp angle pi*k*k/n without
  reduction (optics/fft.go), so its error grows with the length.
"""
import numpy as np
import pytest

import oracle as O
from gpu_util import exact_centroid, rel_l2


def tilted_gauss(n, dx, wl, theta=0.02):
    x = (np.arange(n) - n / 2) * dx
    r2 = x[None, :] ** 2 + x[:, None] ** 2
    w = n * dx / 6
    return np.exp(-r2 / (w * w)) * np.exp(1j * 2 * np.pi / wl * np.sin(theta) * x[None, :])


@pytest.mark.parametrize("method", ["asm_shift", "asm_shift_pad"])
def test_shift_hook_with_own_centroid_is_propagate(method):
    """propagate_shift_at given the oracle's own centroid is propagate, bit for bit."""
    n, dx, wl, z = 64, 2e-6, 632.8e-9, 5e-3
    ex = tilted_gauss(n, dx, wl)
    a = O.Field(ex.copy(), dx)
    O.propagate(a, z, method, O.Context(wavelength=wl))
    b = O.Field(ex.copy(), dx)
    O.propagate_shift_at(b, z, method, O.Context(wavelength=wl), *O.spectral_centroid(O.Field(ex.copy(), dx)))
    assert np.array_equal(a.ex, b.ex)


def test_exact_centroid_agrees_with_the_sequential_sum():
    n, dx, wl = 128, 2e-6, 632.8e-9
    ex = tilted_gauss(n, dx, wl)
    fx, fy = O.spectral_centroid(O.Field(ex.copy(), dx))
    ex_fx, ex_fy = exact_centroid(ex, None, dx)
    assert abs(fx - ex_fx) <= 1e-13 * abs(ex_fx)
    assert abs(fy - ex_fy) <= 1e-13 * abs(ex_fx)


@pytest.mark.parametrize("method", ["asm_shift", "asm_shift_pad"])
def test_shift_output_amplifies_the_centroid_rounding(method):
    """At 128^2 and z = 5 cm the last-bits difference between the two
    centroids moves the output by more than 1e-12 (measured 3.2e-11 and
    1.7e-11): the reference's own floor on these methods."""
    n, dx, wl, z = 128, 2e-6, 632.8e-9, 5e-2
    ex = tilted_gauss(n, dx, wl)
    a = O.Field(ex.copy(), dx)
    O.propagate(a, z, method, O.Context(wavelength=wl))
    b = O.Field(ex.copy(), dx)
    O.propagate_shift_at(b, z, method, O.Context(wavelength=wl), *exact_centroid(ex, None, dx))
    d = rel_l2(a.ex, b.ex)
    assert 1e-12 < d < 1e-9


def test_shift_output_steps_with_the_centroid_bits():
    """Moving the centroid by a few ulps changes the output in steps of
    ~1e-12 (the rounding of the phase flips in some bins), not in proportion."""
    n, dx, wl, z = 64, 2e-6, 632.8e-9, 5e-3
    ex = tilted_gauss(n, dx, wl)
    cx, cy = exact_centroid(ex, None, dx)
    outs = []
    for k in (0, 2, 16):
        f = O.Field(ex.copy(), dx)
        O.propagate_shift_at(f, z, "asm_shift", O.Context(wavelength=wl), cx + k * np.spacing(cx), cy)
        outs.append(f.ex)
    d2, d16 = rel_l2(outs[1], outs[0]), rel_l2(outs[2], outs[0])
    assert 1e-13 < d2 < 1e-11 and 1e-13 < d16 < 1e-10 and d16 < 8 * d2


@pytest.mark.parametrize("n,lo,hi", [(100, 1e-15, 1e-13), (1000, 5e-14, 1e-12), (3000, 2e-13, 2e-12)])
def test_bluestein_error_grows_with_length(n, lo, hi):
    """The oracle's (the reference's) Bluestein line against numpy's FFT: its
    error grows about linearly in n (measured 1.6e-14, 1.7e-13, 5.2e-13)."""
    i = np.arange(n, dtype=np.float64)
    src = np.sin(i * 0.01) + 1j * np.cos(i * 0.017)
    e = rel_l2(O.fft1d(src), np.fft.fft(src))
    assert lo < e < hi


def test_power_of_two_line_is_at_rounding():
    i = np.arange(4096, dtype=np.float64)
    src = np.sin(i * 0.01) + 1j * np.cos(i * 0.017)
    assert rel_l2(O.fft1d(src), np.fft.fft(src)) < 2e-15
