"""GPU parity of the FFT core and of Propagate (every method) against the FP64 oracle.

Mirrors the reference's GPU tests (optics/gpu_test.go:44-158: GPU vs CPU for
2-D sizes {8..128, 12, 27, 100}, 1-D {1024, 4096, 1000, 2049}, whole ASM /
ASM-pad steps) with tighter tolerances: relative L2 <= 1e-12 for the FP64
kernels and <= 1e-5 for the FP32 kernels (FP64 phase arguments).
"""
import math

import numpy as np
import pytest

import oracle as O
from gpu_util import TOL_FP32, TOL_FP64, exact_centroid, log_parity, rel_l2, tol, tol_case, wos
from wos_testutil import (SimpleRNG, analytic_gaussian_fresnel, centroid_x, ref_field,
                          single_bin_plane_wave)

pytestmark = pytest.mark.gpu

PRECS = [pytest.param(wos.FP64, id="fp64"), pytest.param(wos.FP32, id="fp32")]


@pytest.fixture(scope="module", params=PRECS)
def gpu(request):
    g = wos.GPU(request.param)
    yield g
    g.close()


@pytest.fixture(scope="module")
def gpu64():
    g = wos.GPU(wos.FP64)
    yield g
    g.close()


@pytest.fixture(scope="module")
def gpu32():
    g = wos.GPU(wos.FP32)
    yield g
    g.close()


# ------------------------------------------------------------------- FFT
@pytest.mark.parametrize("n", [8, 16, 32, 64, 128, 12, 27, 100, 256, 1024])
def test_fft2d_matches_oracle(gpu, n):
    """gpu_test.go:44-75: forward and round trip."""
    src = ref_field(n, 1.3)
    cpu = O.fft2d(src)
    g = gpu.fft2d(src)
    assert rel_l2(g, cpu) <= tol(gpu.precision)
    back = gpu.fft2d(g, inverse=True)
    assert rel_l2(back, src) <= tol(gpu.precision)


@pytest.mark.parametrize("shape", [(12, 40), (64, 8), (100, 30), (48, 80), (3, 5)])
def test_fft2d_rectangular(gpu, shape):
    a = SimpleRNG(sum(shape)).complex_array(shape)
    assert rel_l2(gpu.fft2d(a), O.fft2d(a)) <= tol(gpu.precision)
    assert rel_l2(gpu.fft2d(a, inverse=True), O.fft2d(a, inverse=True)) <= tol(gpu.precision)


@pytest.mark.parametrize("n", [1024, 4096, 1000, 2049, 2, 3, 17])
def test_fft1d_matches_oracle(gpu, n):
    """gpu_test.go:77-108."""
    i = np.arange(n, dtype=np.float64)
    src = np.sin(i * 0.01) + 1j * np.cos(i * 0.017)
    cpu = O.fft1d(src)
    g = gpu.fft1d(src)
    assert rel_l2(g, cpu) <= tol(gpu.precision)
    assert rel_l2(gpu.fft1d(g, inverse=True), src) <= tol(gpu.precision)


def test_fft_impulse_and_parseval(gpu):
    """fft_test.go:29-60 on the GPU."""
    a = np.zeros((32, 32), complex); a[0, 0] = 1
    assert np.max(np.abs(gpu.fft2d(a) - 1)) <= (1e-12 if gpu.precision == wos.FP64 else 1e-6)
    b = SimpleRNG(7).complex_array((128, 128))
    p1 = np.sum(np.abs(b) ** 2); p2 = np.sum(np.abs(gpu.fft2d(b)) ** 2)
    assert abs(p2 - p1 * 128 * 128) / (p1 * 128 * 128) <= (1e-12 if gpu.precision == wos.FP64 else 1e-6)


# ------------------------------------------------------------- Propagate
def lens_beam(ny, nx, dx, wl, w=200e-6, r_ap=400e-6, f=0.2):
    """Config-1 input: Gaussian clipped by a circular aperture, times a thin-lens phase."""
    x = (np.arange(nx) - nx / 2) * dx
    y = (np.arange(ny) - ny / 2) * dx
    r2 = x[None, :] ** 2 + y[:, None] ** 2
    u = np.exp(-r2 / (w * w)) * (r2 <= r_ap * r_ap)
    return (u * np.exp(-1j * np.pi * r2 / (wl * f))).astype(np.complex128)


def random_phase(ny, nx, seed=1):
    rng = np.random.default_rng(seed)
    return np.exp(1j * rng.uniform(0, 2 * np.pi, (ny, nx)))


def tilted_gauss(ny, nx, dx, wl, w, theta):
    x = (np.arange(nx) - nx / 2) * dx
    y = (np.arange(ny) - ny / 2) * dx
    r2 = x[None, :] ** 2 + y[:, None] ** 2
    return np.exp(-r2 / (w * w)) * np.exp(1j * 2 * np.pi / wl * np.sin(theta) * x[None, :])


CASES = [
    # (ny, nx, dx, wl, z, field)
    (64, 64, 2e-6, 632.8e-9, 5e-3, "lens"),
    (128, 128, 2e-6, 632.8e-9, 5e-2, "lens"),
    (100, 100, 4e-6, 632.8e-9, 1e-2, "lens"),
    (48, 80, 1e-6, 532e-9, 2e-4, "random"),
    (64, 64, 0.25e-6, 1e-6, 1e-6, "random"),     # evanescent bins present
    (96, 60, 3e-6, 633e-9, -4e-3, "lens"),       # backward
    (98, 70, 2e-6, 632.8e-9, 5e-3, "lens"),      # factors of 7: Bluestein lines
]


def make_field(kind, ny, nx, dx, wl, polarized=False):
    if kind == "lens":
        ex = lens_beam(ny, nx, dx, wl, w=min(ny, nx) * dx / 5, r_ap=min(ny, nx) * dx / 3)
    elif kind == "random":
        ex = random_phase(ny, nx)
    else:
        ex = tilted_gauss(ny, nx, dx, wl, min(ny, nx) * dx / 6, 0.02)
    ey = (0.5j * ex) if polarized else None
    return ex, ey


def check_warnings(gctx, octx, exact):
    assert set(gctx.warnings) == set(octx.warnings), (gctx.warnings, octx.warnings)
    for k, (cnt, val) in octx.warnings.items():
        gc, gv = gctx.warnings[k]
        assert gc == cnt, k
        if val != 0:
            assert abs(gv - val) <= (1e-9 if exact else 1e-4) * abs(val) + 1e-300, (k, gv, val)


@pytest.mark.parametrize("method", ["asm", "asm_pad", "asm_shift", "asm_shift_pad", "fresnel_tf",
                                    "fresnel_ir", "fraunhofer"])
@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("polarized", [False, True])
def test_propagate_matches_oracle(gpu, method, case, polarized):
    ny, nx, dx, wl, z, kind = CASES[case]
    if method == "fraunhofer" and ny != nx:
        with pytest.raises(wos.WosError):
            ex, ey = make_field(kind, ny, nx, dx, wl, polarized)
            gpu.propagate(wos.Field(ex, dx, ey), z, method, wos.Context(wavelength=wl))
        return
    if method in ("asm_shift", "asm_shift_pad") and kind == "lens":
        kind = "tilt"
    ex, ey = make_field(kind, ny, nx, dx, wl, polarized)
    of = O.Field(ex.copy(), dx, None if ey is None else ey.copy())
    oc = O.Context(wavelength=wl)
    O.propagate(of, z, method, oc)
    gf = wos.Field(ex.copy(), dx, None if ey is None else ey.copy())
    gc = wos.Context(wavelength=wl)
    gd = gpu.propagate(gf, z, method, gc)
    t = tol_case(gpu.precision, method, ny, nx)
    name = f"propagate {method} {ny}x{nx} {kind}{' pol' if polarized else ''}"
    if method in ("asm_shift", "asm_shift_pad") and gpu.precision == wos.FP64:
        # The output depends on the last bits of the spectral centroid: they
        # decide how the phase k z sqrt(1 - rho^2) of the shifted bins rounds,
        # a phase of ~1e4 rad whose ulp is ~2e-12 rad (two ulps of the
        # centroid move the 64^2 tilted field by 1.3e-12), and the reference
        # sums the centroid in sequence.  So: the GPU's
        # centroid is the exactly summed one to a few ulps; given that
        # centroid the oracle's propagation is the GPU's to the plain FP64
        # bound; against the plain oracle the bound grows by what the
        # oracle's own centroid moves its output (`floor`).  The centroid's
        # rounding scale is eps times the power-weighted mean |f| (sums that
        # cancel leave a small centroid with the absolute error of big sums).
        cx, cy, fs = exact_centroid(ex, ey, dx, with_scale=True)
        ulp = np.finfo(float).eps * max(fs, abs(cx), abs(cy))
        assert abs(gd.centroid_fx - cx) <= 8 * ulp and abs(gd.centroid_fy - cy) <= 8 * ulp, \
            ((gd.centroid_fx - cx) / ulp, (gd.centroid_fy - cy) / ulp)
        xf = O.Field(ex.copy(), dx, None if ey is None else ey.copy())
        O.propagate_shift_at(xf, z, method, O.Context(wavelength=wl), gd.centroid_fx, gd.centroid_fy)
        floor = rel_l2(xf.ex, of.ex)
        given_err = rel_l2(gf.ex, xf.ex)
        log_parity(name + " (GPU centroid)", gpu.precision, given_err, t)
        assert given_err <= t, (given_err, floor)
        if polarized:
            assert rel_l2(gf.ey, xf.ey) <= t
        t = t + max(floor, rel_l2(xf.ey, of.ey) if polarized else 0.0)
    err = rel_l2(gf.ex, of.ex)
    log_parity(name, gpu.precision, err, t)
    assert err <= t, (err, gc.warnings, oc.warnings)
    if polarized:
        assert rel_l2(gf.ey, of.ey) <= t
    assert abs(gf.dx - of.dx) <= 1e-15 * of.dx
    check_warnings(gc, oc, gpu.precision == wos.FP64)


@pytest.mark.parametrize("policy", ["zero", "limit", "tikhonov"])
def test_evanescent_policies(gpu, policy):
    """asmTF branches (propagate.go:159-199) on a field with evanescent content."""
    n, dx, wl = 64, 0.25e-6, 1e-6
    ex = random_phase(n, n, 3)
    z = -2e-6 if policy == "tikhonov" else 2e-6
    kw = dict(wavelength=wl)
    if policy == "zero":
        kw["evanescent"] = "zero"
    elif policy == "limit":
        kw["evanescent_limit"] = 2.0
    else:
        kw.update(backward_regularize=True, tikhonov_alpha=1e-3)
    of = O.Field(ex.copy(), dx); oc = O.Context(**kw)
    O.propagate(of, z, "asm", oc)
    gf = wos.Field(ex.copy(), dx); gc = wos.Context(**kw)
    gpu.propagate(gf, z, "asm", gc)
    assert rel_l2(gf.ex, of.ex) <= tol(gpu.precision)
    check_warnings(gc, oc, gpu.precision == wos.FP64)


def test_z_zero_is_identity(gpu):
    ex = random_phase(32, 32)
    f = wos.Field(ex.copy(), 1e-6)
    gpu.propagate(f, 0.0, "asm", wos.Context(wavelength=5e-7))
    assert np.array_equal(f.ex, ex)


def test_unknown_method_raises(gpu):
    with pytest.raises(wos.WosError):
        gpu.propagate(wos.Field(random_phase(16, 16), 1e-6), 1e-3, "vectorial_x", wos.Context(wavelength=5e-7))


def test_asm_wrap_warning_gpu(gpu):
    """TestASMWrapWarning (asm_wrap_test.go:14-80) through the GPU path."""
    n, width, wl = 1024, 0.008, 632.8e-9
    for z, fires in ((1.0, True), (0.01, False)):
        of = O.build_source("plane", n, width, wl)
        O.apply_grating(of, "phase_sin", 2e-5, modulation=2.0)
        gf = wos.Field(of.ex.copy(), of.dx)
        oc = O.Context(wavelength=wl)
        O.propagate(of, z, "asm", oc)
        gc = wos.Context(wavelength=wl)
        gpu.propagate(gf, z, "asm", gc)
        assert ("asm_alias_wrap" in gc.warnings) == fires
        check_warnings(gc, oc, gpu.precision == wos.FP64)


# ---------------------------------------------------- analytic known answers
@pytest.mark.parametrize("sx,px", [(0.25, 30), (0.9, 45)])
@pytest.mark.parametrize("method", ["asm", "asm_shift"])
def test_single_bin_plane_wave_exact(gpu, sx, px, method):
    """complex_field_test.go:46-79 (max error 1e-8 in FP64; FP32 at its own rounding)."""
    wl, n = 632.8e-9, 256
    k = 2 * math.pi / wl
    dx = px / (sx / wl * n)
    kz = k * math.sqrt(1 - sx * sx)
    for zz in (5e-4, -5e-4):
        f = wos.Field(single_bin_plane_wave(n, dx, wl, sx, 0), dx)
        gpu.propagate(f, zz, method, wos.Context(wavelength=wl))
        x = (np.arange(n) - n / 2) * dx
        want = np.exp(1j * (k * sx * x + kz * zz))[None, :]
        assert np.max(np.abs(f.ex - want)) <= (1e-8 if gpu.precision == wos.FP64 else 2e-5)


@pytest.mark.parametrize("z", [0.005, 0.05, 0.3])
@pytest.mark.parametrize("method", ["asm", "asm_pad", "fresnel_tf"])
def test_gaussian_matches_analytic_fresnel(gpu, z, method):
    """complex_field_test.go:114-139."""
    wl, n, width, w0 = 632.8e-9, 256, 0.004, 5e-4
    dx = width / n
    x = (np.arange(n) - n / 2) * dx
    ex = np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / (w0 * w0)).astype(complex)
    f = wos.Field(ex, dx)
    gpu.propagate(f, z, method, wos.Context(wavelength=wl))
    assert rel_l2(f.ex, analytic_gaussian_fresnel(n, dx, wl, z, w0)) <= 2e-3


def test_asm_shift_centroid(gpu):
    """asm_accuracy_test.go:86-105: asm_shift lands on z*tan(theta)."""
    n, width, wl, theta, z = 512, 0.01, 632.8e-9, 0.005, 0.2
    of = O.build_source("gaussian", n, width, wl, waist=1e-3, tilt_x=theta)
    f = wos.Field(of.ex.copy(), of.dx)
    gpu.propagate(f, z, "asm_shift", wos.Context(wavelength=wl))
    assert abs(centroid_x(f) - z * math.tan(theta)) <= 2e-6


def test_power_conservation(gpu):
    """propagate_test.go:95-111: |P_out - P_in| / P_in <= 1e-6 (energy conservation)."""
    n, width, wl = 512, 0.005, 532e-9
    of = O.build_source("gaussian", n, width, wl, waist=5e-4)
    p0 = of.power()
    for z in (0.01, 0.1, 0.5, 1.5):
        f = wos.Field(of.ex.copy(), of.dx)
        d = gpu.propagate(f, z, "asm", wos.Context(wavelength=wl))
        assert abs(f.power() - p0) / p0 <= 1e-6
        assert abs(d.p_out - d.p_in) / d.p_in <= 1e-6
        # FP32 sees the input rounded to complex64
        assert abs(d.p_in - p0) / p0 <= (1e-12 if gpu.precision == wos.FP64 else 1e-6)


@pytest.mark.parametrize("n", [1536, 2000, 3000, 3600, 6000])
def test_fft1d_long_mixed_radix_lines(gpu, n):
    """2^a 3^b 5^c lines up to 6000 points (one CTA per line, passes between two
    shared-memory buffers) against numpy's FFT; FP64 6000 takes 16 values per
    thread so that its 375 threads fit a CTA."""
    rng = np.random.default_rng(n)
    a = rng.normal(size=n) + 1j * rng.normal(size=n)
    got = gpu.fft1d(a)
    want = np.fft.fft(a)
    assert rel_l2(got, want) <= (1e-12 if gpu.precision == wos.FP64 else 2e-6)
    back = gpu.fft1d(got, inverse=True)
    assert rel_l2(back, a) <= (1e-12 if gpu.precision == wos.FP64 else 2e-6)


def test_fft1d_line_beyond_one_cta_is_unsupported(gpu):
    """4500 = 2^2 3^2 5^3 divides only by E = 4 (1125 threads, more than a CTA
    holds) and its Bluestein length 16384 exceeds the on-chip limit: a clear
    WOS_UNSUPPORTED_SIZE, not a failed launch."""
    with pytest.raises(wos.WosError) as e:
        gpu.fft1d(np.ones(4500, complex))
    assert e.value.status == 2


@pytest.mark.parametrize("n", [100, 768, 1000, 1500, 2000, 3000, 2049])
def test_fp64_lines_are_closer_to_the_exact_dft_than_the_reference(n):
    """The complex128 transforms of lengths that are not powers of two against
    the exact DFT (numpy's pocketfft, double precision), beside the oracle,
    which restates the reference's Bluestein transform (optics/fft.go:159-204):
    the reference forms the chirp angle pi k^2 / n without reducing k^2 mod
    2n, so its error grows with n (~1.7e-16 n), while these lines reduce the
    angle exactly (mixed radix 2/3/5 below 8192 points, else Bluestein).  This
    is the floor that the FP64 parity of non-power-of-two grids sits on."""
    rng = np.random.default_rng(n)
    a = rng.normal(size=n) + 1j * rng.normal(size=n)
    exact = np.fft.fft(a)
    with wos.GPU(wos.FP64) as g:
        got = g.fft1d(a.copy())
    ref = O.fft1d(a)
    e_gpu, e_ref = rel_l2(got, exact), rel_l2(ref, exact)
    log_parity(f"fft1d {n} vs exact DFT", wos.FP64, e_gpu, 1e-14, reference_vs_exact=e_ref)
    assert e_gpu <= 1e-14
    assert e_gpu <= e_ref
