"""Anisotropic propagation on the GPU against the oracle: PropagateUniaxial
(optics/birefringent.go:19-61, two spectral filters) and PropagateAnisotropic
(optics/berreman.go, a Berreman 4x4 eigen-solve per spectral component).
Tolerances: uniaxial as the propagation parity (FP64 1e-12 / 5e-12 on
non-power-of-two grids, FP32 1e-5); Berreman FP64 1e-10 (Durand-Kerner roots
and adjugate null vectors of each component, with CUDA's exp/sincos beside
the host's), FP32 1e-5."""
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


def _f(ny, nx, seed):
    rng = np.random.default_rng(seed)
    return (rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx)),
            rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx)))


@pytest.mark.parametrize("shape,dx,z", [((64, 64), 1e-6, 30e-6), ((48, 80), 0.3e-6, 4e-6), ((64, 64), 0.3e-6, -3e-6)])
@pytest.mark.parametrize("pol", [False, True])
def test_uniaxial_matches_oracle(gpu, shape, dx, z, pol):
    ny, nx = shape
    ex, ey = _f(ny, nx, 1)
    wl, no, ne = 1e-6, 1.5, 1.65
    of = O.Field(ex.copy(), dx, ey.copy() if pol else None)
    O.propagate_uniaxial(of, z, no, ne, O.Context(wavelength=wl))
    gf = wos.Field(ex.copy(), dx, ey.copy() if pol else None)
    gpu.propagate_uniaxial(gf, z, no, ne, wos.Context(wavelength=wl))
    t = tol_case(gpu.precision, "asm", ny, nx)
    assert rel_l2(gf.ex, of.ex) <= t
    if pol:
        assert rel_l2(gf.ey, of.ey) <= t


EPS_BIAXIAL = np.array([[2.30 + 0.01j, 0.05, 0.02],
                        [0.05, 2.25 + 0.005j, 0.0],
                        [0.02, 0.0, 2.20]], dtype=complex)


@pytest.mark.parametrize("shape,dx", [((32, 32), 1e-6), ((24, 40), 0.5e-6)])
def test_berreman_matches_oracle(gpu, shape, dx):
    ny, nx = shape
    ex, ey = _f(ny, nx, 2)
    wl, z = 1e-6, 15e-6
    of = O.Field(ex.copy(), dx, ey.copy())
    O.propagate_anisotropic(of, z, EPS_BIAXIAL, O.Context(wavelength=wl))
    gf = wos.Field(ex.copy(), dx, ey.copy())
    gpu.propagate_anisotropic(gf, z, EPS_BIAXIAL, wos.Context(wavelength=wl))
    t = 1e-10 if gpu.precision == wos.FP64 else 1e-5
    assert rel_l2(gf.ex, of.ex) <= t
    assert rel_l2(gf.ey, of.ey) <= t


def test_berreman_uniaxial_tensor_equals_uniaxial_in_xz_plane(gpu):
    """eps = diag(ne^2, no^2, no^2), field constant along y: the Berreman
    result equals the uniaxial transfer functions (exact for ky = 0)."""
    n, dx, wl, z, no, ne = 64, 1e-6, 1e-6, 20e-6, 1.5, 1.7
    rng = np.random.default_rng(5)
    ex = np.tile(rng.normal(size=n) + 1j * rng.normal(size=n), (n, 1))
    ey = np.tile(rng.normal(size=n) + 1j * rng.normal(size=n), (n, 1))
    fb = wos.Field(ex.copy(), dx, ey.copy())
    gpu.propagate_anisotropic(fb, z, np.diag([ne ** 2, no ** 2, no ** 2]).astype(complex), wos.Context(wavelength=wl))
    fu = wos.Field(ex.copy(), dx, ey.copy())
    gpu.propagate_uniaxial(fu, z, no, ne, wos.Context(wavelength=wl))
    t = 1e-9 if gpu.precision == wos.FP64 else 1e-5
    assert rel_l2(fb.ex, fu.ex) <= t
    assert rel_l2(fb.ey, fu.ey) <= t


def test_anisotropic_argument_errors(gpu):
    ex, ey = _f(16, 16, 3)
    with pytest.raises(wos.WosError):
        gpu.propagate_uniaxial(wos.Field(ex, 1e-6), 1e-6, -1.5, 1.6, wos.Context(wavelength=1e-6))
    with pytest.raises(wos.WosError):
        gpu.propagate_anisotropic(wos.Field(ex, 1e-6, ey), 1e-6, EPS_BIAXIAL, wos.Context(wavelength=0.0))
