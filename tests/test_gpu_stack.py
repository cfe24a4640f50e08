"""Diffractive stack on the GPU: phase masks with split-step BPM segments
between them, the loss sum (|u|^2 - T)^2 and its gradient by the adjoint
chain (wos_bpm_stack_loss_grad / _dev, wos_splitstep_adjoint_dev).  No
reference counterpart: parity is against the oracle's FP64 restatement
(oracle/wos_oracle.c or_bpm_stack_loss_grad, whose adjoint is pinned against
central finite differences on the CPU), against FP64 central differences of
the GPU loss, and between the specialised and general sweeps.

Tolerances: FP64 loss 1e-11 and gradient 1e-10 relative (hundreds of FFT
sweeps); FP32 loss 1e-4 and gradient 1e-3 against the FP64 oracle."""
import numpy as np
import pytest

import oracle as O
from gpu_util import rel_l2, wos

pytestmark = pytest.mark.gpu

PRECS = [pytest.param(wos.FP64, id="fp64"), pytest.param(wos.FP32, id="fp32")]
WL = 633e-9


@pytest.fixture(scope="module", params=PRECS)
def gpu(request):
    g = wos.GPU(request.param)
    yield g
    g.close()


def _tol(prec):
    return (1e-11, 1e-10) if prec == wos.FP64 else (1e-4, 1e-3)


def _medium(graded=True):
    o, g = O.IndexDesc(), wos.IndexDesc()
    for d in (o, g):
        d.re_bg, d.im_bg = 1.5, 2e-6
        if graded:
            d.core_dn, d.core_w, d.core_x0 = 0.01, 20e-6, 3e-6
            d.border_px, d.border_order, d.border_strength = 6, 2, 4e-3
    return o, g


def _case(ny, nx, nl, seed=5):
    rng = np.random.default_rng(seed)
    yy, xx = np.meshgrid(np.arange(ny) - ny / 2, np.arange(nx) - nx / 2, indexing="ij")
    a = np.exp(-(xx ** 2 + yy ** 2) / (min(ny, nx) / 3) ** 2).astype(complex)
    phis = rng.uniform(0, 2 * np.pi, (nl, ny, nx))
    T = rng.uniform(0, 1, (ny, nx)) * np.mean(np.abs(a) ** 2)
    return a, phis, T


def _run(gpu, a, phis, T, dx, zseg, steps, desc, want_grad=True):
    return gpu.bpm_stack_loss_grad(a, phis, T, dx, zseg, steps, desc, wos.Context(wavelength=WL), want_grad)


@pytest.mark.parametrize("shape", [(48, 48), (64, 40), (256, 256)])
def test_bpm_stack_matches_oracle(gpu, shape):
    ny, nx = shape
    a, phis, T = _case(ny, nx, 3)
    dx, zseg, steps = 1e-6, 30e-6, 4
    od, gd = _medium()
    lo, go = O.bpm_stack_loss_grad(a, phis, T, dx, zseg, steps, od, O.Context(wavelength=WL))
    lg, gg = _run(gpu, a, phis, T, dx, zseg, steps, gd)
    tl, tg = _tol(gpu.precision)
    assert abs(lg - lo) <= tl * abs(lo)
    assert rel_l2(gg, go) <= tg


def test_bpm_stack_specialised_equals_general(gpu):
    """256^2 runs the specialised sweeps (screen inside the row sweep); the
    general sweeps give the same loss and gradient."""
    a, phis, T = _case(256, 256, 2, seed=8)
    dx, zseg, steps = 1e-6, 40e-6, 5
    _, gd = _medium()
    l1, g1 = _run(gpu, a, phis, T, dx, zseg, steps, gd)
    gpu.set_fast_path(0)
    try:
        l0, g0 = _run(gpu, a, phis, T, dx, zseg, steps, gd)
    finally:
        gpu.set_fast_path(1)
    fp64 = gpu.precision == wos.FP64
    assert abs(l1 - l0) <= (1e-12 if fp64 else 1e-5) * abs(l0)
    assert rel_l2(g1, g0) <= (1e-11 if fp64 else 1e-4)


def test_bpm_stack_gradient_matches_central_differences():
    """FP64 GPU gradient against central differences (h = 1e-6) of the FP64
    GPU loss on random pixels of every layer."""
    with wos.GPU(wos.FP64) as g:
        a, phis, T = _case(64, 64, 3, seed=2)
        dx, zseg, steps = 1e-6, 25e-6, 3
        _, gd = _medium()
        _, grad = _run(g, a, phis, T, dx, zseg, steps, gd)
        rng = np.random.default_rng(2)
        h, scale = 1e-6, np.max(np.abs(grad))
        for _ in range(24):
            l, j, i = rng.integers(0, 3), rng.integers(0, 64), rng.integers(0, 64)
            p = phis.copy()
            p[l, j, i] += h
            lp, _ = _run(g, a, p, T, dx, zseg, steps, gd, want_grad=False)
            p[l, j, i] -= 2 * h
            lm, _ = _run(g, a, p, T, dx, zseg, steps, gd, want_grad=False)
            assert abs((lp - lm) / (2 * h) - grad[l, j, i]) <= 1e-6 * scale


def test_bpm_stack_fp32_gradient_matches_fp64_adjoint(gpu):
    if gpu.precision == wos.FP64:
        pytest.skip("compares the FP32 context with an FP64 one")
    a, phis, T = _case(256, 256, 3, seed=4)
    dx, zseg, steps = 2e-6, 50e-6, 6
    _, gd = _medium(graded=False)
    l32, g32 = _run(gpu, a, phis, T, dx, zseg, steps, gd)
    with wos.GPU(wos.FP64) as g64:
        l64, gr64 = _run(g64, a, phis, T, dx, zseg, steps, gd)
    assert abs(l32 - l64) <= 1e-4 * abs(l64)
    assert rel_l2(g32, gr64) <= 1e-3


@pytest.mark.parametrize("n", [48, 256])
def test_splitstep_adjoint_inner_product(gpu, n):
    """<A x, y> == <x, A^H y> for the BPM segment and its adjoint."""
    import torch
    rng = np.random.default_rng(n)
    x = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    y = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    dx, z, steps = 1e-6, 30e-6, 4
    _, gd = _medium()
    ctx = wos.Context(wavelength=WL, warnings_enabled=False)
    dt = torch.complex128 if gpu.precision == wos.FP64 else torch.complex64
    xd = torch.from_numpy(x).to(dt).cuda().contiguous()
    yd = torch.from_numpy(y).to(dt).cuda().contiguous()
    torch.cuda.synchronize()
    gpu.split_step_dev(n, n, dx, 1, xd.data_ptr(), z, gd, steps, ctx)
    gpu.split_step_adjoint_dev(n, n, dx, 1, yd.data_ptr(), z, gd, steps, ctx)
    gpu.synchronize()
    ax = xd.cpu().numpy().astype(complex)
    ahy = yd.cpu().numpy().astype(complex)
    lhs, rhs = np.vdot(y, ax), np.vdot(ahy, x)
    scale = np.linalg.norm(ax) * np.linalg.norm(y)
    assert abs(lhs - rhs) <= (1e-12 if gpu.precision == wos.FP64 else 1e-5) * scale


def test_bpm_stack_device_entry_point_matches_host(gpu):
    import torch
    n, nl = 256, 3
    a, phis, T = _case(n, n, nl, seed=6)
    dx, zseg, steps = 1e-6, 30e-6, 4
    _, gd = _medium()
    lh, gh = _run(gpu, a, phis, T, dx, zseg, steps, gd)
    dt = torch.complex128 if gpu.precision == wos.FP64 else torch.complex64
    ad = torch.from_numpy(a).to(dt).cuda()
    pd = torch.from_numpy(phis).cuda()
    td = torch.from_numpy(T).cuda()
    grd = torch.zeros((nl, n, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx = wos.Context(wavelength=WL)
    ld = gpu.bpm_stack_loss_grad_dev(ad.data_ptr(), pd.data_ptr(), td.data_ptr(), grd.data_ptr(), nl, n, n, dx, zseg,
                                     steps, gd, ctx)
    gpu.synchronize()
    fp64 = gpu.precision == wos.FP64
    assert abs(ld - lh) <= (1e-12 if fp64 else 1e-6) * abs(lh)
    assert rel_l2(grd.cpu().numpy(), gh) <= (1e-12 if fp64 else 1e-5)
    l0 = gpu.bpm_stack_loss_grad_dev(ad.data_ptr(), pd.data_ptr(), td.data_ptr(), None, nl, n, n, dx, zseg, steps,
                                     gd, ctx)
    assert abs(l0 - ld) <= 1e-12 * abs(ld)


def test_bpm_stack_argument_errors(gpu):
    a, phis, T = _case(32, 32, 1)
    _, gd = _medium(False)
    with pytest.raises(wos.WosError):
        gpu.bpm_stack_loss_grad(a, phis, T, 1e-6, 1e-5, 0, gd, wos.Context(wavelength=WL))
    with pytest.raises(wos.WosError):
        gpu.bpm_stack_loss_grad(a, phis, T, 1e-6, 1e-5, 2, gd, wos.Context(wavelength=0.0))


@pytest.mark.parametrize("pol", [False, True])
def test_backward_bpm_host_entry_point_is_the_adjoint(gpu, pol):
    """<A x, y> == <x, A^H y> through the host pair split_step / split_step_adjoint."""
    n, dx, z, steps = 64, 1e-6, 25e-6, 5
    rng = np.random.default_rng(12)
    c = lambda: rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))  # noqa: E731
    x, y = c(), c()
    x2, y2 = (c(), c()) if pol else (None, None)
    _, gd = _medium()
    ctx = wos.Context(wavelength=WL, warnings_enabled=False)
    fx = wos.Field(x.copy(), dx, None if x2 is None else x2.copy())
    gpu.split_step(fx, z, gd, steps, ctx)
    fy = wos.Field(y.copy(), dx, None if y2 is None else y2.copy())
    gpu.split_step_adjoint(fy, z, gd, steps, ctx)
    lhs = np.vdot(y, fx.ex) + (np.vdot(y2, fx.ey) if pol else 0)
    rhs = np.vdot(fy.ex, x) + (np.vdot(fy.ey, x2) if pol else 0)
    scale = np.linalg.norm(fx.ex) * np.linalg.norm(y) * (2 if pol else 1)
    assert abs(lhs - rhs) <= (1e-12 if gpu.precision == wos.FP64 else 1e-5) * scale
