"""Size limits: the largest grid the on-chip line transforms take (8192 points
per line, FP32 and FP64) checked through size-independent properties (an
ASM step there and back is the identity for a band-limited field, power is
conserved when no component is evanescent), thin grids against the oracle, and
a clear WOS_UNSUPPORTED_SIZE past the limit."""
import numpy as np
import pytest

import oracle as O
from gpu_util import rel_l2, tol_case, wos

pytestmark = pytest.mark.gpu

PRECS = [pytest.param(wos.FP64, id="fp64"), pytest.param(wos.FP32, id="fp32")]


@pytest.fixture(scope="module", params=PRECS)
def gpu(request):
    g = wos.GPU(request.param)
    yield g
    g.close()


def _beam(n, dx, wl):
    x = (np.arange(n) - n / 2) * dx
    r2 = x[None, :] ** 2 + x[:, None] ** 2
    w = n * dx / 8
    return np.exp(-r2 / w ** 2) * np.exp(-1j * np.pi * r2 / (wl * 0.5))


def test_largest_grid_round_trip_and_power(gpu):
    n, dx, wl, z = 8192, 2e-6, 632.8e-9, 2e-2   # lambda / (2 dx) < 1: nothing evanescent
    ex = _beam(n, dx, wl)
    f = wos.Field(ex.copy(), dx)
    ctx = wos.Context(wavelength=wl)
    d = gpu.propagate(f, z, "asm", ctx)
    assert abs(d.p_out / d.p_in - 1) <= (1e-12 if gpu.precision == wos.FP64 else 1e-6)
    assert "evanescent_filtered" not in ctx.warnings
    gpu.propagate(f, -z, "asm", wos.Context(wavelength=wl))
    assert rel_l2(f.ex, ex) <= (1e-11 if gpu.precision == wos.FP64 else 2e-5)


@pytest.mark.parametrize("shape", [(2, 4096), (4096, 2), (6, 2048)])
def test_thin_grids_match_oracle(gpu, shape):
    ny, nx = shape
    rng = np.random.default_rng(ny * 7 + nx)
    ex = rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))
    dx, wl, z = 1e-6, 632.8e-9, 3e-4
    of = O.Field(ex.copy(), dx)
    O.propagate(of, z, "asm", O.Context(wavelength=wl))
    f = wos.Field(ex.copy(), dx)
    gpu.propagate(f, z, "asm", wos.Context(wavelength=wl))
    assert rel_l2(f.ex, of.ex) <= tol_case(gpu.precision, "asm", ny, nx)


@pytest.mark.parametrize("shape", [(2, 16384), (16384, 2)])
def test_beyond_the_line_limit_is_unsupported(gpu, shape):
    f = wos.Field(np.ones(shape, complex), 1e-6)
    with pytest.raises(wos.WosError) as e:
        gpu.propagate(f, 1e-3, "asm", wos.Context(wavelength=632.8e-9))
    assert e.value.status == 2
