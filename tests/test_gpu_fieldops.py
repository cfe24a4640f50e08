"""GPU parity of the field operations and the 1-D propagator against the oracle:
Field.ApplyJones / ScaleAmplitude / ApplyTilt / ApplyBandlimit / ShiftField
(optics/field.go:109-168,199-228,264-294), diffuserEl.Apply
(optics/elements.go:722-783) and Propagate1D (optics/propagate.go:718-738).

Tolerances: pointwise element arithmetic is FP64 in both context precisions
(bit-identical products; 1e-13 where CUDA's sincos/exp meet the host libm);
the FFT filters and Propagate1D run in the context precision and take the
propagation tolerances (FP64 1e-12, 5e-12 on non-power-of-two lengths; FP32
1e-5)."""
import numpy as np
import pytest

import oracle as O
from gpu_util import TOL_FP32, rel_l2, tol_case, wos

pytestmark = pytest.mark.gpu

PRECS = [pytest.param(wos.FP64, id="fp64"), pytest.param(wos.FP32, id="fp32")]


@pytest.fixture(scope="module", params=PRECS)
def gpu(request):
    g = wos.GPU(request.param)
    yield g
    g.close()


def _field(ny=64, nx=64, pol=False, seed=3):
    rng = np.random.default_rng(seed)
    ex = rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))
    ey = (rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))) if pol else None
    return ex, ey


def _pair(ex, ey, dx):
    of = O.Field(ex.copy(), dx, None if ey is None else ey.copy())
    gf = wos.Field(ex.copy(), dx, None if ey is None else ey.copy())
    return of, gf


# ------------------------------------------------------------ pointwise
@pytest.mark.parametrize("case", ["scalar_diag", "scalar_to_vector", "full"])
def test_jones_matches_oracle(gpu, case):
    pol = case == "full"
    ex, ey = _field(pol=pol)
    a, b, c, d = 0.8 - 0.1j, 0.3j, -0.2 + 0.5j, 0.6 + 0.2j
    if case == "scalar_diag":
        b, c, d = 0, 0, a
    of, gf = _pair(ex, ey, 2e-6)
    O.apply_jones(of, a, b, c, d)
    gpu.apply_jones(gf, a, b, c, d)
    assert gf.polarized == of.polarized == (case != "scalar_diag")
    assert np.array_equal(gf.ex, of.ex)
    if of.polarized:
        assert np.array_equal(gf.ey, of.ey)


@pytest.mark.parametrize("pol", [False, True])
def test_scale_amplitude_matches_oracle(gpu, pol):
    ex, ey = _field(pol=pol)
    of, gf = _pair(ex, ey, 2e-6)
    O.scale_amplitude(of, 0.7 - 1.3j)
    gpu.scale_amplitude(gf, 0.7 - 1.3j)
    assert np.array_equal(gf.ex, of.ex)
    if pol:
        assert np.array_equal(gf.ey, of.ey)


@pytest.mark.parametrize("pol", [False, True])
def test_tilt_matches_oracle(gpu, pol):
    # rows longer than one accumulation chunk (1024 pixels); phases of
    # hundreds of radians, where the running sum's rounding shows
    ex, ey = _field(ny=24, nx=2500, pol=pol)
    of, gf = _pair(ex, ey, 1e-6)
    tx, ty, wl = np.deg2rad(3.0), np.deg2rad(-1.2), 532e-9
    O.apply_tilt(of, tx, ty, wl)
    gpu.apply_tilt(gf, tx, ty, wl)
    assert rel_l2(gf.ex, of.ex) <= 1e-13
    if pol:
        assert rel_l2(gf.ey, of.ey) <= 1e-13


# ------------------------------------------------------------ FFT filters
@pytest.mark.parametrize("shape", [(64, 64), (48, 80), (98, 70)])
@pytest.mark.parametrize("pol", [False, True])
def test_bandlimit_matches_oracle(gpu, shape, pol):
    ny, nx = shape
    ex, ey = _field(ny, nx, pol)
    of, gf = _pair(ex, ey, 2e-6)
    O.apply_bandlimit(of, 0.6, 0.05)
    gpu.apply_bandlimit(gf, 0.6, 0.05)
    t = tol_case(gpu.precision, "asm", ny, nx)
    assert rel_l2(gf.ex, of.ex) <= t
    if pol:
        assert rel_l2(gf.ey, of.ey) <= t
    # disabled options leave the field untouched
    g2 = wos.Field(ex.copy(), 2e-6)
    gpu.apply_bandlimit(g2, 1.0, 0.05)
    gpu.apply_bandlimit(g2, 0.0, 0.05)
    assert np.array_equal(g2.ex, ex)


@pytest.mark.parametrize("shape", [(64, 64), (48, 80), (98, 70)])
@pytest.mark.parametrize("pol", [False, True])
def test_shift_field_matches_oracle(gpu, shape, pol):
    ny, nx = shape
    dx = 2e-6
    ex, ey = _field(ny, nx, pol)
    of, gf = _pair(ex, ey, dx)
    O.shift_field(of, 3.3 * dx, -1.7 * dx)
    gpu.shift_field(gf, 3.3 * dx, -1.7 * dx)
    t = tol_case(gpu.precision, "asm", ny, nx)
    assert rel_l2(gf.ex, of.ex) <= t
    if pol:
        assert rel_l2(gf.ey, of.ey) <= t


def test_shift_field_whole_pixels_is_a_roll(gpu):
    ex, _ = _field(64, 48)
    dx = 1e-6
    gf = wos.Field(ex.copy(), dx)
    gpu.shift_field(gf, 5 * dx, -3 * dx)
    want = np.roll(np.roll(ex, 5, axis=1), -3, axis=0)
    assert rel_l2(gf.ex, want) <= (1e-13 if gpu.precision == wos.FP64 else TOL_FP32)


# ------------------------------------------------------------ diffuser
@pytest.mark.parametrize("corr", [0.0, 2e-5])
@pytest.mark.parametrize("pol", [False, True])
def test_diffuser_matches_oracle(gpu, corr, pol):
    ex, ey = _field(64, 96, pol)
    dx = 2e-6
    of, gf = _pair(ex, ey, dx)
    args = (np.pi / 2, corr, 0.9, 7, 13e-6, -5e-6)
    O.apply_diffuser(of, *args)
    gpu.apply_diffuser(gf, *args)
    # no correlation filter: FP64 pointwise work in both precisions
    t = 1e-13 if corr == 0 else tol_case(gpu.precision, "asm", 64, 96)
    assert rel_l2(gf.ex, of.ex) <= t
    if pol:
        assert rel_l2(gf.ey, of.ey) <= t


def test_diffuser_screen_statistics(gpu):
    """The transmission is amp exp(i phase) with the phase rescaled to
    standard deviation sigma (elements.go:763-781)."""
    n, dx, sigma = 128, 2e-6, 0.8
    gf = wos.Field(np.ones((n, n), complex), dx)
    gpu.apply_diffuser(gf, sigma, 1e-5, 0.5, 11, 0.0, 0.0)
    assert np.allclose(np.abs(gf.ex), 0.5, atol=1e-12)
    ph = np.angle(gf.ex)
    ph = ph - np.angle(np.mean(np.exp(1j * ph)))
    assert abs(np.std(np.angle(np.exp(1j * ph))) - sigma) < 0.1


# ------------------------------------------------------------ Propagate1D
@pytest.mark.parametrize("n", [256, 100, 98])
@pytest.mark.parametrize("z", [4e-5, -2e-5])
@pytest.mark.parametrize("evanescent", ["decay", "zero"])
def test_propagate1d_matches_oracle(gpu, n, z, evanescent):
    rng = np.random.default_rng(n)
    a = rng.normal(size=n) + 1j * rng.normal(size=n)
    dx, wl = 0.4e-6, 1e-6          # lambda / (2 dx) > 1: evanescent bins present
    octx = O.Context(wavelength=wl, evanescent=evanescent)
    gctx = wos.Context(wavelength=wl, evanescent=evanescent)
    want = O.propagate1d(a, dx, z, wl, octx)
    got = gpu.propagate1d(a, dx, z, wl, gctx)
    assert rel_l2(got, want) <= tol_case(gpu.precision, "asm", 1 if n == 256 else n, n)
    assert set(gctx.warnings) == set(octx.warnings)
    for k, (cnt, val) in octx.warnings.items():
        assert gctx.warnings[k][0] == cnt
        assert abs(gctx.warnings[k][1] - val) <= (1e-7 if gpu.precision == wos.FP64 else 1e-3) * abs(val)


def test_propagate1d_plane_wave_kat(gpu):
    """A single-bin plane wave picks up exactly H(f_m) (propagate1d_test.go:8-35)."""
    n, dx, wl, z, m = 512, 1e-6, 632.8e-9, 1e-3, 37
    x = (np.arange(n) - n / 2) * dx
    a = np.exp(2j * np.pi * m * x / (n * dx))
    got = gpu.propagate1d(a, dx, z, wl)
    fx = m / (n * dx)
    h = np.exp(1j * 2 * np.pi / wl * z * np.sqrt((1 - wl * fx) * (1 + wl * fx)))
    assert rel_l2(got, a * h) <= (1e-12 if gpu.precision == wos.FP64 else 1e-5)


def test_propagate1d_argument_errors(gpu):
    with pytest.raises(wos.WosError):
        gpu.propagate1d(np.ones(1, complex), 1e-6, 1e-3, 632.8e-9)
    with pytest.raises(wos.WosError):
        gpu.propagate1d(np.ones(64, complex), 1e-6, 1e-3, 0.0)
