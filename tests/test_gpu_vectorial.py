"""GPU vector angular spectrum (wos_propagate_vectorial) against the oracle's
restatement of PropagateVectorial (optics/vectorial.go:14-80).  Tolerances:
FP64 1e-12 (5e-12 on non-power-of-two grids), FP32 1e-5, per component."""
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


CASES = [
    # (ny, nx, dx, wl, z, policy)
    (64, 64, 1e-6, 633e-9, 2e-4, "decay"),
    (64, 64, 0.4e-6, 1e-6, 3e-6, "decay"),       # evanescent bins
    (48, 80, 0.4e-6, 1e-6, 2e-6, "zero"),
    (64, 64, 0.4e-6, 1e-6, -2e-6, "reg"),        # backward, Tikhonov
    (98, 70, 1e-6, 633e-9, -1e-4, "decay"),      # Bluestein lines, backward (zeroed)
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_vectorial_matches_oracle(gpu, case):
    ny, nx, dx, wl, z, policy = CASES[case]
    rng = np.random.default_rng(case)
    ex = rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))
    ey = rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))
    kw = dict(evanescent="zero") if policy == "zero" else {}
    if policy == "reg":
        kw = dict(backward_regularize=True, tikhonov_alpha=1e-2)
    of = O.Field(ex.copy(), dx, ey.copy())
    ez_o = O.propagate_vectorial(of, z, O.Context(wavelength=wl, **kw))
    gf = wos.Field(ex.copy(), dx, ey.copy())
    ez_g = gpu.propagate_vectorial(gf, z, wos.Context(wavelength=wl, **kw))
    t = tol_case(gpu.precision, "asm", ny, nx)
    assert rel_l2(gf.ex, of.ex) <= t
    assert rel_l2(gf.ey, of.ey) <= t
    assert rel_l2(ez_g, ez_o) <= t


def test_vectorial_uses_ey_of_a_scalar_field(gpu):
    """Like the reference (which reads f.Ey whatever Polarized says), the Ey
    buffer of a scalar field takes part; z == 0 changes nothing."""
    n, dx, wl = 32, 1e-6, 633e-9
    rng = np.random.default_rng(9)
    ex = rng.normal(size=(n, n)) + 0j
    f = wos.Field(ex.copy(), dx)          # polarized = False, ey = zeros
    ez = gpu.propagate_vectorial(f, 0.0, wos.Context(wavelength=wl))
    assert np.array_equal(f.ex, ex) and not ez.any()
    of = O.Field(ex.copy(), dx)
    ez_o = O.propagate_vectorial(of, 1e-4, O.Context(wavelength=wl))
    ez_g = gpu.propagate_vectorial(f, 1e-4, wos.Context(wavelength=wl))
    assert rel_l2(ez_g, ez_o) <= tol_case(gpu.precision, "asm", n, n)
