"""Pins the FP64 oracle against the reference's own known-answer tests.

The reference (Go package `optics`) holds no stored golden vectors: every
expectation in its test files is analytic or CPU-vs-GPU.  Each test below is
one of those known-answer tests, restated against the oracle with the same
inputs and tolerances (file:line of the Go test in each docstring).
"""
import math

import numpy as np
import pytest

import oracle as O
from wos_testutil import (SimpleRNG, analytic_gaussian_fresnel, centroid_x, complex_normal,
                          evanescent_field, far_field_radius, naive_dft, rel_l2,
                          single_bin_plane_wave, waist_radius)


def ctx_for(wl):
    """ctxFor, optics/propagate_test.go:8-10."""
    return O.Context(wavelength=wl, evanescent="decay")


# ---------------------------------------------------------------- fft_test.go
def test_fft_round_trip():
    """TestFFTRoundTrip, fft_test.go:10-26."""
    n = 64
    a = SimpleRNG(42).complex_array((n, n))
    b = O.fft2d(O.fft2d(a), inverse=True)
    assert np.max(np.abs(b - a)) <= 1e-12


def test_fft_impulse():
    """TestFFTImpulse, fft_test.go:29-39."""
    n = 32
    a = np.zeros((n, n), complex); a[0, 0] = 1
    assert np.max(np.abs(O.fft2d(a) - 1)) <= 1e-12


def test_fft_parseval():
    """TestFFTParseval, fft_test.go:42-60."""
    n = 128
    a = SimpleRNG(7).complex_array((n, n))
    p1 = np.sum(np.abs(a) ** 2)
    p2 = np.sum(np.abs(O.fft2d(a)) ** 2)
    assert abs(p2 - p1 * n * n) / (p1 * n * n) <= 1e-12


def test_fft_matches_numpy_pow2_and_bluestein():
    """Spectrum of the restated FFT against an independent FFT (numpy pocketfft)."""
    for n in (8, 16, 64, 12, 27, 100):
        a = SimpleRNG(n).complex_array((n, n))
        assert rel_l2(O.fft2d(a), np.fft.fft2(a)) < 1e-13
        assert rel_l2(O.fft2d(a, inverse=True), np.fft.ifft2(a)) < 1e-13
    a = SimpleRNG(3).complex_array((12, 40))
    assert rel_l2(O.fft2d(a), np.fft.fft2(a)) < 1e-13


# ------------------------------------------------------- asm_improve_test.go
@pytest.mark.parametrize("n", [100, 200, 480])
def test_bluestein_matches_naive_dft(n):
    """TestBluesteinMatchesNaiveDFT, asm_improve_test.go:23-38 (one RNG stream over n)."""
    rng = SimpleRNG(99)
    for m in (100, 200, 480):
        a = rng.complex_array((m,))
        if m == n:
            break
    want = naive_dft(a)
    assert np.max(np.abs(O.fft1d(a) - want)) <= 1e-9


def test_bluestein_round_trip():
    """TestBluesteinRoundTrip, asm_improve_test.go:40-56."""
    a = SimpleRNG(5).complex_array((100,))
    b = O.fft1d(O.fft1d(a), inverse=True)
    assert np.max(np.abs(b - a)) <= 1e-12


def test_fft2d_non_power_of_two():
    """TestFFT2DNonPowerOfTwo, asm_improve_test.go:58-83."""
    n = 100
    a = SimpleRNG(11).complex_array((n, n))
    assert np.max(np.abs(O.fft2d(O.fft2d(a), inverse=True) - a)) <= 1e-11
    b = np.zeros((n, n), complex); b[0, 0] = 1
    assert np.max(np.abs(O.fft2d(b) - 1)) <= 1e-11


def test_asm_non_power_of_two_grid():
    """TestASMNonPowerOfTwoGrid, asm_improve_test.go:87-107."""
    n, width, wl = 100, 0.01, 632.8e-9
    f = O.build_source("plane", n, width, wl)
    p0 = f.power()
    z = 0.3
    O.propagate(f, z, "asm", ctx_for(wl))
    want = 2 * math.pi / wl * z
    c = f.ex[n // 2, n // 2]
    got = math.remainder(math.atan2(c.imag, c.real) - want, 2 * math.pi)
    assert abs(got) <= 1e-6
    assert abs(f.power() - p0) / p0 <= 1e-6


def test_asm_shift_pad_moderate_tilt():
    """TestASMShiftPadModerateTilt, asm_improve_test.go:131-150."""
    n, width, wl, theta, z = 512, 0.01, 632.8e-9, 0.005, 0.2
    ref = O.build_source("gaussian", n, width, wl, waist=1e-3, tilt_x=theta)
    O.propagate(ref, z, "asm", ctx_for(wl))
    sp = O.build_source("gaussian", n, width, wl, waist=1e-3, tilt_x=theta)
    O.propagate(sp, z, "asm_shift_pad", ctx_for(wl))
    assert rel_l2(sp.ex, ref.ex) <= 1e-3
    assert abs(centroid_x(sp) - z * math.tan(theta)) <= 2e-6


@pytest.mark.slow
def test_asm_shift_pad_walk_off():
    """TestASMShiftPadWalkOff, asm_improve_test.go:154-165."""
    n, width, wl, waist, theta, z = 1024, 0.01, 632.8e-9, 1e-3, 0.03, 0.15
    f = O.build_source("gaussian", n, width, wl, waist=waist, tilt_x=theta)
    O.propagate(f, z, "asm_shift_pad", ctx_for(wl))
    assert abs(centroid_x(f) - z * math.tan(theta)) <= 3e-4


def test_evanescent_limit_truncation():
    """TestEvanescentLimitTruncation, asm_improve_test.go:182-210."""
    n, dx, wl, q, z = 256, 0.25e-6, 1e-6, 96, 1e-6
    f0 = q / (n * dx)
    assert wl * f0 > 1
    decay = (2 * math.pi / wl) * z * math.sqrt((wl * f0) ** 2 - 1)
    fd = O.Field(evanescent_field(n, dx, q), dx)
    O.propagate(fd, z, "asm", ctx_for(wl))
    assert abs(abs(fd.ex[0, 0]) - math.exp(-decay)) <= 1e-6
    fl = O.Field(evanescent_field(n, dx, q), dx)
    O.propagate(fl, z, "asm", O.Context(wavelength=wl, evanescent_limit=1.0))
    assert fl.power() <= 1e-20


def test_backward_tikhonov():
    """TestBackwardTikhonov, asm_improve_test.go:215-253."""
    n, width, wl, z = 256, 0.01, 632.8e-9, 0.05
    f = O.build_source("gaussian", n, width, wl, waist=1e-3)
    orig = f.clone()
    O.propagate(f, z, "asm", ctx_for(wl))
    cb = O.Context(wavelength=wl, backward_regularize=True, tikhonov_alpha=1e-3)
    O.propagate(f, -z, "asm", cb)
    assert rel_l2(f.ex, orig.ex) <= 1e-6
    assert "backward_regularized" in cb.warnings
    nE, dx, wlE = 256, 0.25e-6, 1e-6
    ev = O.Field(evanescent_field(nE, dx, 96), dx)
    O.propagate(ev, -1e-6, "asm", O.Context(wavelength=wlE, backward_regularize=True,
                                             tikhonov_alpha=1e-3))
    assert np.all(np.isfinite(ev.ex)) and ev.power() > 0
    ez = O.Field(evanescent_field(nE, dx, 96), dx)
    c = ctx_for(wlE)
    O.propagate(ez, -1e-6, "asm", c)
    assert np.all(np.isfinite(ez.ex)) and ez.power() <= 1e-20
    assert "backward_evanescent" in c.warnings


# ----------------------------------------------------- complex_field_test.go
@pytest.mark.parametrize("sx,px", [(0.25, 30), (0.9, 45)])
@pytest.mark.parametrize("method", ["asm", "asm_shift"])
def test_tilted_plane_wave_single_bin_exact(sx, px, method):
    """TestTiltedPlaneWaveSingleBinExact, complex_field_test.go:46-79."""
    wl, n = 632.8e-9, 256
    k = 2 * math.pi / wl
    dx = px / (sx / wl * n)
    z = 5e-4
    kz = k * math.sqrt(1 - sx * sx)
    for zz in (z, -z):
        f = O.Field(single_bin_plane_wave(n, dx, wl, sx, 0), dx)
        O.propagate(f, zz, method, ctx_for(wl))
        x = (np.arange(n) - n / 2) * dx
        want = np.exp(1j * (k * sx * x + kz * zz))[None, :]
        assert np.max(np.abs(f.ex - want)) <= 1e-8


@pytest.mark.parametrize("z", [0.005, 0.05, 0.3])
@pytest.mark.parametrize("method", ["asm", "asm_pad", "fresnel_tf"])
def test_asm_gaussian_matches_analytic_complex(z, method):
    """TestASMGaussianMatchesAnalyticComplex, complex_field_test.go:114-139."""
    wl, n, width, w0 = 632.8e-9, 256, 0.004, 5e-4
    dx = width / n
    x = (np.arange(n) - n / 2) * dx
    ex = np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / (w0 * w0)).astype(complex)
    want = analytic_gaussian_fresnel(n, dx, wl, z, w0)
    g = O.Field(ex, dx)
    O.propagate(g, z, method, ctx_for(wl))
    assert rel_l2(g.ex, want) <= 2e-3


def test_fraunhofer_complex_field_exact():
    """TestFraunhoferComplexFieldExact, complex_field_test.go:144-181."""
    wl, n, width, w0, z = 632.8e-9, 256, 0.002, 1e-4, 20.0
    dx = width / n
    x = (np.arange(n) - n / 2) * dx
    ex = np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / (w0 * w0)).astype(complex)
    k = 2 * math.pi / wl
    dxo = wl * z / (n * dx)
    xo = (np.arange(n) - n / 2) * dxo
    r2 = xo[None, :] ** 2 + xo[:, None] ** 2
    s = math.pi * w0 * np.sqrt(r2) / (wl * z)
    want = np.exp(1j * k * z) / complex(0, wl * z) * np.exp(1j * k * r2 / (2 * z)) * (math.pi * w0 * w0) * np.exp(-s * s)
    g = O.Field(ex, dx)
    O.propagate(g, z, "fraunhofer", ctx_for(wl))
    assert rel_l2(g.ex, want) <= 1e-3
    assert abs(g.dx - dxo) <= 1e-18


@pytest.mark.parametrize("z,want", [(0.1, True), (50.0, False)])
def test_fraunhofer_nearfield_warning(z, want):
    """TestFraunhoferNearfieldWarningMeasuresInput, complex_field_test.go:186-219."""
    wl, n, width, w0 = 632.8e-9, 256, 0.002, 2e-4
    dx = width / n
    x = (np.arange(n) - n / 2) * dx
    ex = np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / (w0 * w0)).astype(complex)
    c = O.Context(wavelength=wl)
    O.propagate(O.Field(ex, dx), z, "fraunhofer", c)
    assert ("fraunhofer_nearfield" in c.warnings) == want


def test_asm_pad_shift_variants_complex_agree():
    """TestASMPadShiftVariantsComplexAgree, complex_field_test.go:222-248."""
    wl, n, width, z = 632.8e-9, 256, 0.01, 0.1
    ref = O.build_source("gaussian", n, width, wl, waist=1e-3, tilt_x=0.002)
    O.propagate(ref, z, "asm", ctx_for(wl))
    for m in ("asm_pad", "asm_shift", "asm_shift_pad"):
        g = O.build_source("gaussian", n, width, wl, waist=1e-3, tilt_x=0.002)
        O.propagate(g, z, m, ctx_for(wl))
        assert rel_l2(g.ex, ref.ex) <= 1e-6, m


# ------------------------------------------------------- propagate_test.go
def test_plane_wave_phase():
    """TestPlaneWavePhase, propagate_test.go:13-35."""
    n, width, wl, z = 256, 0.01, 632.8e-9, 0.3
    f = O.build_source("plane", n, width, wl)
    O.propagate(f, z, "asm", ctx_for(wl))
    c = f.ex[n // 2, n // 2]
    got = math.remainder(math.atan2(c.imag, c.real) - 2 * math.pi / wl * z, 2 * math.pi)
    assert abs(got) <= 1e-6
    I = f.intensity()
    assert np.max(np.abs(I - I[0, 0])) <= 1e-12 * I[0, 0]


@pytest.mark.slow
def test_tilted_beam_shift():
    """TestTiltedBeamShift, propagate_test.go:39-63."""
    n, width, wl, theta, z = 1024, 0.01, 632.8e-9, 0.002, 0.3
    f = O.build_source("gaussian", n, width, wl, waist=1e-3, tilt_x=theta)
    O.propagate(f, z, "asm", ctx_for(wl))
    assert abs(centroid_x(f) - z * math.tan(theta)) <= 2e-6


@pytest.mark.slow
def test_gaussian_waist_evolution():
    """TestGaussianWaistEvolution, propagate_test.go:66-92."""
    n, width, wl, w0, z = 1024, 0.01, 632.8e-9, 3e-4, 0.4
    f = O.build_source("gaussian", n, width, wl, waist=w0)
    O.propagate(f, z, "asm", ctx_for(wl))
    zr = math.pi * w0 * w0 / wl
    want = w0 * math.sqrt(1 + (z / zr) ** 2)
    assert abs(waist_radius(f) - want) / want <= 0.01


def test_power_conservation_asm():
    """TestPowerConservationASM, propagate_test.go:95-111."""
    n, width, wl = 512, 0.005, 532e-9
    f = O.build_source("gaussian", n, width, wl, waist=5e-4)
    p0 = f.power()
    for z in (0.01, 0.1, 0.5, 1.5):
        g = f.clone()
        O.propagate(g, z, "asm", ctx_for(wl))
        assert abs(g.power() - p0) / p0 <= 1e-6


@pytest.mark.slow
def test_fresnel_matches_asm():
    """TestFresnelMatchesASM, propagate_test.go:115-137."""
    n, width, wl, z = 1024, 0.01, 633e-9, 0.15
    f = O.build_source("gaussian", n, width, wl, waist=5e-4, tilt_x=0.002)
    ref = f.clone(); O.propagate(ref, z, "asm", ctx_for(wl))
    g = f.clone(); O.propagate(g, z, "fresnel_tf", ctx_for(wl))
    assert rel_l2(g.ex, ref.ex) <= 0.01


def test_fresnel_ir_matches_asm():
    """TestFresnelIRMatchesASM, propagate_test.go:144-202."""
    n, dx, wl, w0, z = 256, 4e-6, 632.8e-9, 100e-6, 0.05
    assert z >= n * dx * dx / wl
    x = (np.arange(n) - n / 2) * dx
    ex = np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / (w0 * w0)).astype(complex)
    ref = O.Field(ex.copy(), dx); O.propagate(ref, z, "asm", ctx_for(wl))
    g = O.Field(ex.copy(), dx); O.propagate(g, z, "fresnel_ir", ctx_for(wl))
    assert rel_l2(g.ex, ref.ex) <= 1e-4
    bright = np.abs(ref.ex) >= 0.2 * np.abs(ref.ex).max()
    ph = np.angle(g.ex[bright] / ref.ex[bright])
    d = np.abs(np.remainder(ph - ph[0] + np.pi, 2 * np.pi) - np.pi)
    assert d.max() <= 1e-3


# -------------------------------------------------- asm_accuracy_test.go
def test_asm_pad_agrees_asm_no_wrap():
    """TestASMPadAgreesASMNoWrap, asm_accuracy_test.go:50-64."""
    n, width, wl, z = 512, 0.01, 632.8e-9, 0.2
    ref = O.build_source("gaussian", n, width, wl, waist=1e-3)
    O.propagate(ref, z, "asm", ctx_for(wl))
    pad = O.build_source("gaussian", n, width, wl, waist=1e-3)
    O.propagate(pad, z, "asm_pad", ctx_for(wl))
    assert rel_l2(pad.ex, ref.ex) <= 1e-4


def test_asm_pad_power_conservation():
    """TestASMPadPowerConservation, asm_accuracy_test.go:67-82."""
    n, width, wl = 512, 0.005, 532e-9
    f = O.build_source("gaussian", n, width, wl, waist=5e-4)
    p0 = f.power()
    for z in (0.01, 0.1, 0.5):
        g = f.clone()
        O.propagate(g, z, "asm_pad", ctx_for(wl))
        assert abs(g.power() - p0) / p0 <= 1e-6


def test_asm_shift_matches_asm_moderate_tilt():
    """TestASMShiftMatchesASMModerateTilt, asm_accuracy_test.go:86-105."""
    n, width, wl, theta, z = 512, 0.01, 632.8e-9, 0.005, 0.2
    ref = O.build_source("gaussian", n, width, wl, waist=1e-3, tilt_x=theta)
    O.propagate(ref, z, "asm", ctx_for(wl))
    sh = O.build_source("gaussian", n, width, wl, waist=1e-3, tilt_x=theta)
    O.propagate(sh, z, "asm_shift", ctx_for(wl))
    assert rel_l2(sh.ex, ref.ex) <= 1e-3
    assert abs(centroid_x(sh) - z * math.tan(theta)) <= 2e-6


@pytest.mark.slow
def test_asm_shift_spectral_wrap_accuracy():
    """TestASMShiftSpectralWrapAccuracy, asm_accuracy_test.go:111-130."""
    n, width, wl, waist, theta, z = 1024, 0.01, 632.8e-9, 1e-4, 0.03, 0.05
    want = z * math.tan(theta)
    errs = {}
    for m in ("asm_shift", "asm"):
        f = O.build_source("gaussian", n, width, wl, waist=waist, tilt_x=theta)
        O.propagate(f, z, m, ctx_for(wl))
        errs[m] = abs(centroid_x(f) - want)
    assert errs["asm_shift"] <= 1e-6
    assert errs["asm_shift"] < errs["asm"] / 100


@pytest.mark.slow
def test_asm_pad_walk_off_accuracy():
    """TestASMPadWalkOffAccuracy, asm_accuracy_test.go:135-154."""
    n, width, wl, waist, theta, z = 1024, 0.01, 632.8e-9, 1e-3, 0.03, 0.15
    want = z * math.tan(theta)
    errs = {}
    for m in ("asm_pad", "asm"):
        f = O.build_source("gaussian", n, width, wl, waist=waist, tilt_x=theta)
        O.propagate(f, z, m, ctx_for(wl))
        errs[m] = abs(centroid_x(f) - want)
    assert errs["asm_pad"] <= 3e-4
    assert errs["asm_pad"] < errs["asm"] / 2


# --------------------------------------------------------- medium_test.go
def _uniform(re, im=0.0):
    d = O.IndexDesc()
    d.re_bg, d.im_bg = re, im
    return d


def test_split_step_uniform_index():
    """TestSplitStepUniformIndex, medium_test.go:8-27."""
    n, width, wl, z = 256, 0.01, 632.8e-9, 0.1
    f = O.build_source("plane", n, width, wl)
    p0 = f.power()
    O.splitstep(f, z, _uniform(1.5), 20, ctx_for(wl))
    c = f.ex[n // 2, n // 2]
    got = math.remainder(math.atan2(c.imag, c.real) - 2 * math.pi / wl * 1.5 * z, 2 * math.pi)
    assert abs(got) <= 1e-6
    assert abs(f.power() - p0) / p0 <= 1e-9


def test_split_step_absorption():
    """TestSplitStepAbsorption, medium_test.go:29-43."""
    n, width, wl, nim, z = 256, 0.01, 1e-6, 1e-4, 1e-3
    f = O.build_source("plane", n, width, wl)
    p0 = f.power()
    O.splitstep(f, z, _uniform(1.0, nim), 10, ctx_for(wl))
    want = p0 * math.exp(-2 * (2 * math.pi / wl) * nim * z)
    assert abs(f.power() - want) / want <= 1e-3


def test_split_step_stratified():
    """TestSplitStepStratified, medium_test.go:45-66 (layer z<0.05: n=1.5, else 1)."""
    n, width, wl, z = 256, 0.01, 632.8e-9, 0.1
    f = O.build_source("plane", n, width, wl)
    d = _uniform(1.0)
    d.n_layers = 1
    d.layer_z[0], d.layer_re[0], d.layer_im[0] = 0.05, 1.5, 0.0
    O.splitstep(f, z, d, 20, ctx_for(wl))
    c = f.ex[n // 2, n // 2]
    got = math.remainder(math.atan2(c.imag, c.real) - 2 * math.pi / wl * 0.125, 2 * math.pi)
    assert abs(got) <= 1e-6


# --------------------------------------------- polychromatic / volume tests
def test_polychromatic_plane_wave():
    """TestPolychromaticPlaneWave, polychromatic_test.go:8-26."""
    n, width, wl, z = 256, 0.01, 632.8e-9, 0.05
    f = O.build_source("plane", n, width, wl)
    out = O.polychromatic(f, z, [632.8e-9, 532e-9], [1, 0.5], "asm", ctx_for(wl))
    dx = width / n
    want = 1.5 * (1e-3 / (n * n * dx * dx))
    assert np.max(np.abs(out - want)) <= 1e-9 * want


def test_polychromatic_single_matches_mono():
    """TestPolychromaticSingleMatchesMono, polychromatic_test.go:28-45."""
    n, width, wl, z = 256, 0.01, 632.8e-9, 0.1
    f = O.build_source("gaussian", n, width, wl, waist=1e-3)
    g = f.clone(); O.propagate(g, z, "asm", ctx_for(wl))
    out = O.polychromatic(f, z, [wl], [1], "asm", ctx_for(wl))
    I = g.intensity()
    assert np.all(np.abs(out - I) <= 1e-9 * I)


def test_propagate3d_volume():
    """TestPropagate3DVolume, volume_test.go:8-32."""
    n, width, wl, w0 = 512, 0.01, 632.8e-9, 3e-4
    f = O.build_source("gaussian", n, width, wl, waist=w0)
    p0 = f.power()
    zs = [0.05, 0.1, 0.2, 0.3]
    vol = O.propagate3d(f, zs, "asm", ctx_for(wl))
    zr = math.pi * w0 * w0 / wl
    for q, z in enumerate(zs):
        g = O.Field(vol[q, 0], f.dx)
        want = w0 * math.sqrt(1 + (z / zr) ** 2)
        assert abs(waist_radius(g) - want) / want <= 0.01
    assert abs(f.power() - p0) / p0 <= 1e-12
    v0 = O.propagate3d(f, [0.0], "asm", ctx_for(wl))
    assert np.array_equal(v0[0, 0], f.ex)


# --------------------------------------------------- propagate1d_test.go
def test_propagate1d_plane_wave():
    """TestPropagate1DPlaneWave, propagate1d_test.go:8-34."""
    n, dx, wl, z = 256, 1e-5, 632.8e-9, 0.3
    a = np.ones(n, complex)
    p0 = np.sum(np.abs(a) ** 2)
    b = O.propagate1d(a, dx, z, wl, ctx_for(wl))
    got = math.remainder(math.atan2(b[n // 2].imag, b[n // 2].real) - 2 * math.pi / wl * z, 2 * math.pi)
    assert abs(got) <= 1e-6
    assert abs(np.sum(np.abs(b) ** 2) - p0) / p0 <= 1e-9


def test_propagate1d_gaussian():
    """TestPropagate1DGaussian, propagate1d_test.go:36-67."""
    n, width, wl, w0, z = 512, 0.01, 632.8e-9, 5e-4, 0.4
    dx = width / n
    x = (np.arange(n) - n / 2) * dx
    a = np.exp(-x * x / (w0 * w0)).astype(complex)

    def rms(v):
        w = np.abs(v) ** 2
        return math.sqrt((w * x * x).sum() / w.sum())
    s0 = rms(a)
    b = O.propagate1d(a, dx, z, wl, ctx_for(wl))
    zr = math.pi * w0 * w0 / wl
    got = (rms(b) / s0) ** 2
    want = 1 + (z / zr) ** 2
    assert abs(got - want) / want <= 0.02


# ------------------------------------------------------- asm_wrap_test.go
def test_asm_wrap_warning():
    """TestASMWrapWarning, asm_wrap_test.go:14-80, at the Propagate level: a plane wave on a
    20 um phase_sin grating (modulation 2) on a 1024 / 8 mm grid warns for a 1 m step
    (ratio >= 2) and stays silent for a 10 mm step."""
    n, width, wl = 1024, 0.008, 632.8e-9
    for z, fires in ((1.0, True), (0.01, False)):
        f = O.build_source("plane", n, width, wl)
        O.apply_grating(f, "phase_sin", 2e-5, modulation=2.0)
        c = ctx_for(wl)
        O.propagate(f, z, "asm", c)
        assert ("asm_alias_wrap" in c.warnings) == fires
        if fires:
            assert c.warnings["asm_alias_wrap"][1] >= 2


# ------------------------------------------------------- coherence_test.go
def test_schell_source_coherence():
    """TestSchellSourceCoherence, coherence_test.go:10-40 (harness noise, same statistics)."""
    n, dx, w0, sigc, m = 256, 1e-5, 1e-3, 2e-4, 128
    noise = complex_normal(1, (m, n, n))
    fields = O.schell_realizations(n, dx, w0, sigc, noise)
    for dpx in (1, 2, 4, 8, 16):
        a = fields[:, :, : n - dpx]
        b = fields[:, :, dpx:]
        num = np.sum(a.real * b.real + a.imag * b.imag)
        da = np.sum(np.abs(a) ** 2); db = np.sum(np.abs(b) ** 2)
        got = num / math.sqrt(da * db)
        want = math.exp(-(dpx * dx) ** 2 / (2 * sigc * sigc))
        assert abs(got - want) <= 0.03, (dpx, got, want)


@pytest.mark.slow
def test_schell_far_field():
    """TestSchellFarField, coherence_test.go:45-58 (harness noise)."""
    n, dx, w0, sigc, wl, z, m = 512, 1.25e-5, 1e-3, 3.75e-5, 632.8e-9, 1.0, 160
    noise = complex_normal(2, (m, n, n))
    fields = O.schell_realizations(n, dx, w0, sigc, noise)
    out = np.zeros((m, n, n), complex)
    for q in range(m):
        g = O.Field(fields[q], dx)
        O.propagate(g, z, "fraunhofer", ctx_for(wl))
        out[q] = g.ex
    I = O.average_intensity(out)
    dxo = wl * z / (n * dx)
    got = far_field_radius(I, n, dxo)
    want = (wl * z / math.pi) * math.sqrt(1 / w0 ** 2 + 1 / sigc ** 2)
    assert abs(got - want) / want <= 0.1


# ------------------------------------------------ inverse-design oracle
def test_oracle_gradient_matches_finite_difference():
    """The FP64 adjoint of the oracle agrees with central finite differences (h=1e-6)."""
    n, dx, wl, z = 64, 4e-6, 633e-9, 2e-3
    rng = np.random.default_rng(0)
    phi = rng.uniform(0, 2 * np.pi, (n, n))
    a = np.ones((n, n), complex)
    T = rng.uniform(0, 2, (n, n))
    ctx = O.Context(wavelength=wl)
    _, g = O.asm_phase_loss_grad(a, phi, T, dx, z, ctx)
    h = 1e-6
    for _ in range(8):
        j, i = rng.integers(0, n, 2)
        p1 = phi.copy(); p1[j, i] += h
        p2 = phi.copy(); p2[j, i] -= h
        l1, _ = O.asm_phase_loss_grad(a, p1, T, dx, z, ctx, want_grad=False)
        l2, _ = O.asm_phase_loss_grad(a, p2, T, dx, z, ctx, want_grad=False)
        fd = (l1 - l2) / (2 * h)
        assert abs(fd - g[j, i]) <= 1e-4 * max(1.0, abs(fd)), (fd, g[j, i])


def test_hash_noise01_known_values():
    """hashNoise01 (elements.go:710-720) against an independent 64-bit restatement."""
    M = (1 << 64) - 1
    for (x, y, s) in ((0, 0, 1), (3, -7, 1), (-250, 375, 42), (123456, 654321, 9)):
        h = ((s * 0x9E3779B97F4A7C15) & M) ^ ((x * 0xC2B2AE3D27D4EB4F) & M) ^ ((y * 0x165667B19E3779F9) & M)
        h ^= h >> 30; h = (h * 0xBF58476D1CE4E5B9) & M
        h ^= h >> 27; h = (h * 0x94D049BB133111EB) & M
        h ^= h >> 31
        assert O.hash_noise01(x, y, s) == (h >> 11) / float(1 << 53)


def test_tilt_follows_the_running_sum():
    """The oracle's tilt phase is the reference's running sum, which differs
    from a direct evaluation k (sx x + sy y) in the last bits: the GPU test
    above therefore pins the accumulation order, not just the physics."""
    ny, nx, dx, wl = 4, 2500, 1e-6, 532e-9
    tx = np.deg2rad(3.0)
    f = O.Field(np.ones((ny, nx), complex), dx)
    O.apply_tilt(f, tx, 0.0, wl)
    k = 2 * np.pi / wl
    direct = np.exp(1j * k * np.sin(tx) * f.x(np.arange(nx)))[None, :]
    err = np.max(np.abs(f.ex - direct))
    assert 0 < err < 1e-9


def _stack_case(n=32, nl=2, seed=5):
    rng = np.random.default_rng(seed)
    a = np.exp(-(((np.arange(n) - n / 2)[None, :] ** 2 + (np.arange(n) - n / 2)[:, None] ** 2) / (n / 3) ** 2))
    a = a.astype(complex)
    phis = rng.uniform(0, 2 * np.pi, (nl, n, n))
    T = rng.uniform(0, 1, (n, n))
    d = O.IndexDesc()
    d.re_bg, d.im_bg = 1.5, 1e-6
    d.core_dn, d.core_w = 0.01, 8e-6
    d.border_px, d.border_order, d.border_strength = 4, 2, 5e-3
    return a, phis, T, d


def test_oracle_bpm_stack_gradient_matches_finite_differences():
    """The stack adjoint (conjugate transfer functions and screens, slices
    reversed) is the exact gradient of the forward loss."""
    a, phis, T, d = _stack_case()
    dx, zseg, steps = 1e-6, 20e-6, 3
    ctx = O.Context(wavelength=633e-9)
    loss, g = O.bpm_stack_loss_grad(a, phis, T, dx, zseg, steps, d, ctx)
    rng = np.random.default_rng(9)
    h = 1e-6
    for _ in range(6):
        l, j, i = rng.integers(0, phis.shape[0]), rng.integers(0, 32), rng.integers(0, 32)
        p = phis.copy(); p[l, j, i] += h
        lp, _ = O.bpm_stack_loss_grad(a, p, T, dx, zseg, steps, d, ctx, want_grad=False)
        p[l, j, i] -= 2 * h
        lm, _ = O.bpm_stack_loss_grad(a, p, T, dx, zseg, steps, d, ctx, want_grad=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[l, j, i]) <= 1e-6 * np.max(np.abs(g)), (l, j, i, fd, g[l, j, i])


def test_oracle_bpm_stack_forward_is_masks_and_splitstep():
    a, phis, T, d = _stack_case(n=16, nl=2)
    dx, zseg, steps = 1e-6, 10e-6, 2
    ctx = O.Context(wavelength=633e-9)
    f = O.Field(a.copy(), dx)
    for l in range(2):
        f.ex *= np.exp(1j * phis[l])
        O.splitstep(f, zseg, d, steps, O.Context(wavelength=633e-9))
    want = np.sum((np.abs(f.ex) ** 2 - T) ** 2)
    loss, _ = O.bpm_stack_loss_grad(a, phis, T, dx, zseg, steps, d, ctx, want_grad=False)
    assert abs(loss - want) <= 1e-12 * abs(want)


def test_oracle_vectorial_transverse_matches_scalar_asm():
    """The transverse components of the vector ASM are the scalar ASM step
    (vectorial.go:14-80 and propagate.go:159-181 differ only in rounding)."""
    n, dx, wl, z = 64, 1e-6, 633e-9, 2e-4
    rng = np.random.default_rng(1)
    ex = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    ey = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    fv = O.Field(ex.copy(), dx, ey.copy())
    O.propagate_vectorial(fv, z, O.Context(wavelength=wl))
    fs = O.Field(ex.copy(), dx, ey.copy())
    O.propagate(fs, z, "asm", O.Context(wavelength=wl))
    assert np.linalg.norm(fv.ex - fs.ex) <= 1e-12 * np.linalg.norm(fs.ex)
    assert np.linalg.norm(fv.ey - fs.ey) <= 1e-12 * np.linalg.norm(fs.ey)


def test_oracle_vectorial_field_is_divergence_free():
    """kx Ex + ky Ey + kz Ez = 0 for every propagating plane wave."""
    n, dx, wl, z = 64, 0.5e-6, 633e-9, 3e-6
    rng = np.random.default_rng(2)
    ex = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    ey = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    f = O.Field(ex.copy(), dx, ey.copy())
    ez = O.propagate_vectorial(f, z, O.Context(wavelength=wl))
    i = np.arange(n)
    fx = np.where(i <= n // 2, i, i - n) / (n * dx)   # freq (field.go:297-303): +Nyquist
    FX, FY = np.meshgrid(fx, fx)
    rho = wl * np.hypot(FX, FY)
    prop = rho < 1
    kz = 2 * np.pi / wl * np.sqrt(np.clip(1 - rho ** 2, 0, None))
    div = 2 * np.pi * FX * np.fft.fft2(f.ex) + 2 * np.pi * FY * np.fft.fft2(f.ey) + kz * np.fft.fft2(ez)
    scale = np.abs(2 * np.pi / wl * np.fft.fft2(f.ex)).max()
    assert np.abs(div[prop]).max() <= 1e-10 * scale


def test_oracle_berreman_reduces_to_uniaxial_in_the_xz_plane():
    """For eps = diag(ne^2, no^2, no^2) and a field constant along y (ky = 0,
    where the uniaxial transfer functions are exact) the Berreman 4x4
    propagation equals PropagateUniaxial (berreman.go:9-12)."""
    n, dx, wl, z, no, ne = 64, 1e-6, 1e-6, 20e-6, 1.5, 1.7
    rng = np.random.default_rng(5)
    rowx = rng.normal(size=n) + 1j * rng.normal(size=n)
    rowy = rng.normal(size=n) + 1j * rng.normal(size=n)
    ex = np.tile(rowx, (n, 1))
    ey = np.tile(rowy, (n, 1))
    fb = O.Field(ex.copy(), dx, ey.copy())
    O.propagate_anisotropic(fb, z, np.diag([ne ** 2, no ** 2, no ** 2]).astype(complex), O.Context(wavelength=wl))
    fu = O.Field(ex.copy(), dx, ey.copy())
    O.propagate_uniaxial(fu, z, no, ne, O.Context(wavelength=wl))
    assert np.linalg.norm(fb.ex - fu.ex) <= 1e-9 * np.linalg.norm(fu.ex)
    assert np.linalg.norm(fb.ey - fu.ey) <= 1e-9 * np.linalg.norm(fu.ey)


def test_oracle_uniaxial_isotropic_is_asm_in_the_medium():
    """n_o = n_e = n: both components take the ASM of a medium of index n,
    i.e. the vacuum ASM at wavelength wl / n."""
    n, dx, wl, z, nn = 64, 1e-6, 1e-6, 30e-6, 1.6
    rng = np.random.default_rng(6)
    ex = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    fu = O.Field(ex.copy(), dx)
    O.propagate_uniaxial(fu, z, nn, nn, O.Context(wavelength=wl))
    fa = O.Field(ex.copy(), dx)
    O.propagate(fa, z, "asm", O.Context(wavelength=wl / nn))
    assert np.linalg.norm(fu.ex - fa.ex) <= 1e-10 * np.linalg.norm(fa.ex)
