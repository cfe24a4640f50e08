"""The specialised power-of-two ASM sweeps agree with the general sweeps and
with the oracle, for every launch configuration the autotuner may pick."""
import numpy as np
import pytest

import oracle as O
from gpu_util import rel_l2, tol, wos

pytestmark = pytest.mark.gpu


def field(n, seed=3):
    rng = np.random.default_rng(seed)
    return np.exp(1j * rng.uniform(0, 2 * np.pi, (n, n)))


@pytest.mark.parametrize("prec", [wos.FP64, wos.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("n", [256, 512, 1024, 2048])
def test_fast_equals_general(prec, n):
    dx, wl, z = 2e-6, 632.8e-9, 3e-3
    ex = field(n)
    with wos.GPU(prec) as g:
        a = wos.Field(ex.copy(), dx)
        ca = wos.Context(wavelength=wl)
        g.propagate(a, z, "asm", ca)
        g.set_fast_path(False)
        b = wos.Field(ex.copy(), dx)
        cb = wos.Context(wavelength=wl)
        g.propagate(b, z, "asm", cb)
    assert rel_l2(a.ex, b.ex) <= tol(prec)
    assert ca.warnings.keys() == cb.warnings.keys()
    if n <= 512:
        o = O.Field(ex.copy(), dx)
        O.propagate(o, z, "asm", O.Context(wavelength=wl))
        assert rel_l2(a.ex, o.ex) <= tol(prec)


@pytest.mark.parametrize("prec", [wos.FP64, wos.FP32], ids=["fp64", "fp32"])
def test_every_launch_configuration(prec):
    n, dx, wl, z = 512, 1e-6, 5e-7, 2e-4
    ex = field(n, 4)
    o = O.Field(ex.copy(), dx)
    O.propagate(o, z, "asm", O.Context(wavelength=wl))
    with wos.GPU(prec) as g:
        best = g.autotune(n, n)
        assert best[0] in (8, 16) and best[1] in (8, 16) and best[2] >= 1
        for re in (8, 16):
            for ce in (8, 16):
                for w in (1, 2, 4, 8):
                    try:
                        g.set_tune(n, n, re, ce, w)
                    except wos.WosError:
                        continue
                    f = wos.Field(ex.copy(), dx)
                    g.propagate(f, z, "asm", wos.Context(wavelength=wl))
                    assert rel_l2(f.ex, o.ex) <= tol(prec), (re, ce, w)


@pytest.mark.parametrize("prec", [wos.FP64, wos.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("n", [256, 1024, 2048])
def test_wrap_histogram_fast_equals_general(prec, n):
    """asmWrapWarn's spectral radius (optics/propagate.go:247-310) from the
    histogram binned inside the specialised column sweep equals the general
    sweep's and the oracle's, bin for bin at the 90 % crossing."""
    dx, wl = 2e-6, 632.8e-9
    z = 3.0 * n * dx * 2 * dx / wl      # walk-off test active: z wl / (2 dx) > n dx
    rng = np.random.default_rng(n)
    x = (np.arange(n) - n / 2) * dx
    env = np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / (n * dx / 5) ** 2)
    ex = env * np.exp(1j * rng.uniform(0, 0.6, (n, n)))
    res = []
    with wos.GPU(prec) as g:
        for fast in (True, False):
            g.set_fast_path(fast)
            f = wos.Field(ex.copy(), dx)
            c = wos.Context(wavelength=wl)
            d = g.propagate(f, z, "asm", c)
            assert d.wrap_checked == 1
            res.append((d.spectral_radius, dict(c.warnings), f.ex))
    assert res[0][0] == res[1][0]
    assert res[0][1].keys() == res[1][1].keys()
    assert rel_l2(res[0][2], res[1][2]) <= tol(prec)
    o = O.Field(ex.copy(), dx)
    assert res[0][0] == O.spectral_radius(o, 0.90)


def _dev_propagate(g, prec, ex, ey, dx, z, wl, mode, diag=True):
    """propagate_dev on device buffers of the context precision (the layout the
    pipelined sweeps take), returning the fields and the diagnostics."""
    import torch
    g.set_fast_path(mode)
    dt = torch.complex128 if prec == wos.FP64 else torch.complex64
    comps = [ex] if ey is None else [ex, ey]
    buf = torch.from_numpy(np.stack(comps)).to(dt).cuda().contiguous()
    torch.cuda.synchronize()  # the context's stream does not wait for torch's
    ny, nx = ex.shape
    c = wos.Context(wavelength=wl)
    d = g.propagate_dev(ny, nx, dx, len(comps), buf.data_ptr(), buf.data_ptr(), z, "asm", c, diag=diag)
    g.synchronize()
    return buf.cpu().numpy().astype(np.complex128), d, c


@pytest.mark.parametrize("shape", [(256, 256), (2048, 2048), (256, 1024), (1024, 256)])
@pytest.mark.parametrize("ncomp", [1, 2])
@pytest.mark.parametrize("z", [2e-3, -2e-3])
def test_fp64_h_table_equals_evaluated_h(shape, ncomp, z):
    """Without diagnostics the pipelined complex128 column sweep reads H from
    the table of its FP64 values; the one-shot sweep (mode 2) evaluates H in
    the reference's operation order: the fields agree element for element,
    forward and backward."""
    ny, nx = shape
    dx, wl = 2e-6, 632.8e-9
    rng = np.random.default_rng(ny + 3 * nx + ncomp)
    ex = np.exp(1j * rng.uniform(0, 2 * np.pi, (ny, nx)))
    ey = 0.5 * np.exp(1j * rng.uniform(0, 2 * np.pi, (ny, nx))) if ncomp == 2 else None
    with wos.GPU(wos.FP64) as g:
        a, _, _ = _dev_propagate(g, wos.FP64, ex, ey, dx, z, wl, 1, diag=False)
        b, _, _ = _dev_propagate(g, wos.FP64, ex, ey, dx, z, wl, 2, diag=False)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("prec", [wos.FP64, wos.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("shape", [(256, 256), (512, 512), (1024, 1024), (2048, 2048), (256, 1024), (1024, 256)])
@pytest.mark.parametrize("ncomp", [1, 2])
@pytest.mark.parametrize("mode", [1, 3])
def test_pipelined_equals_one_shot(prec, shape, ncomp, mode):
    """The persistent TMA-pipelined sweeps (mode 1: columns, mode 3: rows and
    columns) compute exactly what the one-shot specialised sweeps (mode 2)
    compute, element for element; the diagnostics differ only in the grouping
    of their partial sums."""
    ny, nx = shape
    dx, wl, z = 2e-6, 632.8e-9, 2e-3
    rng = np.random.default_rng(ny * 7 + nx + ncomp)
    ex = np.exp(1j * rng.uniform(0, 2 * np.pi, (ny, nx)))
    ey = 0.5 * np.exp(1j * rng.uniform(0, 2 * np.pi, (ny, nx))) if ncomp == 2 else None
    with wos.GPU(prec) as g:
        a, da, ca = _dev_propagate(g, prec, ex, ey, dx, z, wl, mode)
        b, db, cb = _dev_propagate(g, prec, ex, ey, dx, z, wl, 2)
    assert np.array_equal(a, b)
    p_exact = ny * nx * dx * dx * (1.25 if ncomp == 2 else 1.0)
    for d in (da, db):
        assert abs(d.p_in - p_exact) <= 1e-6 * p_exact
    assert abs(da.p_in - db.p_in) <= 1e-12 * db.p_in
    assert abs(da.p_out - db.p_out) <= 1e-12 * db.p_out
    assert ca.warnings.keys() == cb.warnings.keys()
    if ny == nx <= 512:
        o = O.Field(ex.copy(), dx)
        O.propagate(o, z, "asm", O.Context(wavelength=wl))
        assert rel_l2(a[0], o.ex) <= tol(prec)


@pytest.mark.parametrize("prec", [wos.FP64, wos.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("mode", [1, 3])
def test_pipelined_wrap_histogram(prec, mode):
    """The alias-wrap histogram accumulated across the tiles of a persistent
    column CTA gives the one-shot kernels' spectral radius and warnings."""
    n, dx, wl = 1024, 2e-6, 632.8e-9
    z = 3.0 * n * dx * 2 * dx / wl
    x = (np.arange(n) - n / 2) * dx
    ex = np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / (n * dx / 5) ** 2).astype(np.complex128)
    with wos.GPU(prec) as g:
        a, da, ca = _dev_propagate(g, prec, ex, None, dx, z, wl, mode)
        b, db, cb = _dev_propagate(g, prec, ex, None, dx, z, wl, 2)
    assert da.wrap_checked == 1 and db.wrap_checked == 1
    assert da.spectral_radius == db.spectral_radius
    assert ca.warnings.keys() == cb.warnings.keys()
    assert np.array_equal(a, b)


def test_fp32_phase_beyond_revolution_range_uses_general_sweep():
    """|z / lambda| >= 2^28 revolutions: the FP32 specialised column sweep
    declines (its exact revolution reduction needs fewer), the general sweep
    with its FP64 Cody-Waite reduction propagates, and the result still meets
    the FP32 tolerance against the oracle."""
    n, dx, wl, z = 256, 40e-6, 500e-9, 150.0  # z / wl = 3e8 > 2^28
    ex = field(n, 9)
    o = O.Field(ex.copy(), dx)
    O.propagate(o, z, "asm", O.Context(wavelength=wl))
    with wos.GPU(wos.FP32) as g:
        f = wos.Field(ex.copy(), dx)
        g.propagate(f, z, "asm", wos.Context(wavelength=wl))
    assert rel_l2(f.ex, o.ex) <= tol(wos.FP32)


@pytest.mark.parametrize("prec", [wos.FP64, wos.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("shape,nf", [((512, 512), 7), ((256, 1024), 4), ((300, 200), 3)])
def test_batch_dev_equals_single_calls(prec, shape, nf):
    """wos_propagate_batch_dev (fields on concurrent streams on the power-of-two
    ASM path, in order otherwise) gives each field exactly what one
    wos_propagate_dev call gives it."""
    import torch
    ny, nx = shape
    dx, wl, z = 2e-6, 632.8e-9, 3e-3
    rng = np.random.default_rng(nf)
    dt = torch.complex128 if prec == wos.FP64 else torch.complex64
    fields = [np.exp(1j * rng.uniform(0, 2 * np.pi, (ny, nx))) for _ in range(nf)]
    with wos.GPU(prec) as g:
        ctx = wos.Context(wavelength=wl, warnings_enabled=False)
        a = [torch.from_numpy(f).to(dt).cuda() for f in fields]
        b = [torch.from_numpy(f).to(dt).cuda() for f in fields]
        outs = [torch.empty_like(x) for x in a]
        torch.cuda.synchronize()
        g.propagate_batch_dev(ny, nx, dx, 1, [x.data_ptr() for x in a], [o.data_ptr() for o in outs], z, "asm", ctx)
        for x in b:
            g.propagate_dev(ny, nx, dx, 1, x.data_ptr(), x.data_ptr(), z, "asm", ctx)
        g.synchronize()
        for o, x in zip(outs, b):
            assert np.array_equal(o.cpu().numpy(), x.cpu().numpy())


@pytest.mark.parametrize("prec", [wos.FP64, wos.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("method", ["asm", "asm_pad", "fraunhofer"])
def test_host_batch_equals_single_calls(prec, method):
    """wos_propagate_batch (uploads, sweeps and downloads of consecutive fields
    overlapped) gives every field, its warnings and its output pitch exactly
    what one wos_propagate call gives."""
    n, dx, wl = 256, 2e-6, 632.8e-9
    z = 0.5 if method == "fraunhofer" else 4e-3
    rng = np.random.default_rng(21)
    srcs = [(np.exp(1j * rng.uniform(0, 2 * np.pi, (n, n))), None if k % 2 else
             0.3j * np.exp(1j * rng.uniform(0, 2 * np.pi, (n, n)))) for k in range(5)]
    with wos.GPU(prec) as g:
        batch = [wos.Field(ex.copy(), dx, None if ey is None else ey.copy()) for ex, ey in srcs]
        cb = wos.Context(wavelength=wl)
        diags = g.propagate_batch(batch, z, method, cb)
        assert len(diags) == len(batch)
        cs = wos.Context(wavelength=wl)
        for (ex, ey), fb in zip(srcs, batch):
            fs = wos.Field(ex.copy(), dx, None if ey is None else ey.copy())
            g.propagate(fs, z, method, cs)
            assert np.array_equal(fs.ex, fb.ex)
            if ey is not None:
                assert np.array_equal(fs.ey, fb.ey)
            assert fs.dx == fb.dx
        assert cb.warnings == cs.warnings
