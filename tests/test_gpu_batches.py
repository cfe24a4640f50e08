"""GPU parity of split-step BPM, the batch entry points (polychromatic, volume,
Gaussian Schell), the thin-element multiply and the inverse-design adjoint,
each against the FP64 oracle on the same seeded inputs (tolerances: rel-L2
<= 1e-12 FP64, <= 1e-5 FP32 unless a test states otherwise), plus the
reference's own known-answer tests for these paths.
"""
import math

import numpy as np
import pytest

import oracle as O
from gpu_util import TOL_FP64, TOL_FP64_SCHELL, rel_l2, tol, tol_case, tol_fp32_splitstep, wos
from wos_testutil import complex_normal, waist_radius

pytestmark = pytest.mark.gpu

PRECS = [pytest.param(wos.FP64, id="fp64"), pytest.param(wos.FP32, id="fp32")]


@pytest.fixture(scope="module", params=PRECS)
def gpu(request):
    g = wos.GPU(request.param)
    yield g
    g.close()


def check_warnings(gctx, octx, exact=True):
    assert set(gctx.warnings) == set(octx.warnings), (gctx.warnings, octx.warnings)
    for k, (cnt, val) in octx.warnings.items():
        gc, gv = gctx.warnings[k]
        assert gc == cnt, (k, gc, cnt)
        if val != 0:
            assert abs(gv - val) <= (1e-7 if exact else 1e-3) * abs(val), (k, gv, val)


def desc_pair(**kw):
    o, g = O.IndexDesc(), wos.IndexDesc()
    for k, v in kw.items():
        if k in ("layer_z", "layer_re", "layer_im"):
            for i, x in enumerate(v):
                getattr(o, k)[i] = x
                getattr(g, k)[i] = x
        else:
            setattr(o, k, v)
            setattr(g, k, v)
    return o, g


# ------------------------------------------------------------------ BPM
def test_split_step_uniform_index_kat(gpu):
    """TestSplitStepUniformIndex (medium_test.go:8-27)."""
    n, width, wl, z = 256, 0.01, 632.8e-9, 0.1
    of = O.build_source("plane", n, width, wl)
    p0 = of.power()
    f = wos.Field(of.ex.copy(), of.dx)
    _, d = desc_pair(re_bg=1.5)
    gpu.split_step(f, z, d, 20, wos.Context(wavelength=wl))
    c = f.ex[n // 2, n // 2]
    got = math.remainder(math.atan2(c.imag, c.real) - 2 * math.pi / wl * 1.5 * z, 2 * math.pi)
    assert abs(got) <= (1e-6 if gpu.precision == wos.FP64 else 1e-4)
    assert abs(f.power() - p0) / p0 <= (1e-9 if gpu.precision == wos.FP64 else 1e-5)


def test_split_step_absorption_kat(gpu):
    """TestSplitStepAbsorption (medium_test.go:29-43)."""
    n, width, wl, nim, z = 256, 0.01, 1e-6, 1e-4, 1e-3
    of = O.build_source("plane", n, width, wl)
    p0 = of.power()
    f = wos.Field(of.ex.copy(), of.dx)
    _, d = desc_pair(re_bg=1.0, im_bg=nim)
    gpu.split_step(f, z, d, 10, wos.Context(wavelength=wl))
    want = p0 * math.exp(-2 * (2 * math.pi / wl) * nim * z)
    assert abs(f.power() - want) / want <= 1e-3


@pytest.mark.parametrize("kind", ["uniform", "stratified", "graded", "graded_pol"])
def test_split_step_matches_oracle(gpu, kind):
    n, dx, wl = 128, 0.5e-6, 1.55e-6
    x = (np.arange(n) - n / 2) * dx
    r2 = (x[None, :] - 5e-6) ** 2 + x[:, None] ** 2
    ex = np.exp(-r2 / (8e-6) ** 2).astype(complex)
    ey = 0.5j * ex if kind == "graded_pol" else None
    if kind == "uniform":
        od, gd = desc_pair(re_bg=1.45, im_bg=1e-5)
        steps, z = 8, 16e-6
    elif kind == "stratified":
        od, gd = desc_pair(re_bg=1.0, n_layers=1, layer_z=[10e-6], layer_re=[1.5], layer_im=[0.0])
        steps, z = 10, 20e-6
    else:
        od, gd = desc_pair(re_bg=1.45, im_bg=1e-5, core_dn=0.01, core_w=25e-6, zmod_amp=0.1,
                           zmod_period=200e-6, border_px=16, border_order=2, border_strength=5e-3)
        steps, z = 12, 24e-6
    of = O.Field(ex.copy(), dx, None if ey is None else ey.copy())
    oc = O.Context(wavelength=wl)
    O.splitstep(of, z, od, steps, oc)
    f = wos.Field(ex.copy(), dx, None if ey is None else ey.copy())
    gc = wos.Context(wavelength=wl)
    gpu.split_step(f, z, gd, steps, gc)
    assert rel_l2(f.ex, of.ex) <= tol(gpu.precision) * 10
    if ey is not None:
        assert rel_l2(f.ey, of.ey) <= tol(gpu.precision) * 10
    check_warnings(gc, oc, gpu.precision == wos.FP64)


def test_split_step_maps_matches_descriptor(gpu):
    """A sampled medium (per-slice maps, as a Go IndexFunc closure would be sampled) gives the
    same field as the parametric descriptor it samples."""
    n, dx, wl, steps, z = 64, 0.5e-6, 1.55e-6, 6, 12e-6
    od, gd = desc_pair(re_bg=1.45, im_bg=1e-5, core_dn=0.01, core_w=10e-6, zmod_amp=0.1,
                       zmod_period=50e-6, border_px=8, border_order=2, border_strength=5e-3)
    dz = z / steps
    re = np.zeros((steps, n, n)); im = np.zeros((steps, n, n))
    for s in range(steps):
        zc = z * s / steps + dz / 2
        re[s], im[s] = O.index_map(od, n, n, dx, zc)
    x = (np.arange(n) - n / 2) * dx
    ex = np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / (6e-6) ** 2).astype(complex)
    a = wos.Field(ex.copy(), dx)
    gpu.split_step(a, z, gd, steps, wos.Context(wavelength=wl))
    b = wos.Field(ex.copy(), dx)
    gpu.split_step_maps(b, z, re, im, steps, wos.Context(wavelength=wl))
    assert rel_l2(b.ex, a.ex) <= tol(gpu.precision)


# ------------------------------------------------------------ polychromatic
def test_polychromatic_plane_wave_kat(gpu):
    """TestPolychromaticPlaneWave (polychromatic_test.go:8-26)."""
    n, width, wl, z = 256, 0.01, 632.8e-9, 0.05
    of = O.build_source("plane", n, width, wl)
    out = gpu.polychromatic(wos.Field(of.ex.copy(), of.dx), z, [632.8e-9, 532e-9], [1, 0.5], "asm",
                            wos.Context(wavelength=wl))
    want = 1.5 * (1e-3 / (n * n * of.dx ** 2))
    assert np.max(np.abs(out - want)) <= (1e-9 if gpu.precision == wos.FP64 else 1e-6) * want


@pytest.mark.parametrize("method", ["asm", "asm_pad", "fresnel_tf"])
def test_polychromatic_matches_oracle(gpu, method):
    n, dx, z = 128, 2e-6, 2e-3
    x = (np.arange(n) - n / 2) * dx
    g = (np.cos(2 * np.pi * x / 20e-6) >= np.cos(np.pi * 0.5)).astype(float)
    ex = np.tile(g, (n, 1)).astype(complex) * np.exp(-(x[:, None] ** 2) / (80e-6) ** 2)
    wls = np.linspace(400e-9, 700e-9, 9)
    ws = np.linspace(0.5, 1.5, 9)
    ref = O.polychromatic(O.Field(ex.copy(), dx), z, wls, ws, method, O.Context(wavelength=wls[0]))
    out = gpu.polychromatic(wos.Field(ex.copy(), dx), z, wls, ws, method, wos.Context(wavelength=wls[0]))
    assert rel_l2(out, ref) <= tol(gpu.precision)


# ------------------------------------------------------------------ volume
def test_volume_kat(gpu):
    """TestPropagate3DVolume (volume_test.go:8-32)."""
    n, width, wl, w0 = 512, 0.01, 632.8e-9, 3e-4
    of = O.build_source("gaussian", n, width, wl, waist=w0)
    zs = [0.05, 0.1, 0.2, 0.3]
    f = wos.Field(of.ex.copy(), of.dx)
    vol = gpu.volume(f, zs, "asm", wos.Context(wavelength=wl))
    zr = math.pi * w0 * w0 / wl
    for q, z in enumerate(zs):
        g = wos.Field(vol[q, 0], of.dx)
        want = w0 * math.sqrt(1 + (z / zr) ** 2)
        assert abs(waist_radius(g) - want) / want <= 0.01
    assert np.array_equal(f.ex, of.ex)


@pytest.mark.parametrize("method", ["asm", "fresnel_tf", "asm_pad"])
def test_volume_matches_oracle(gpu, method):
    n, dx, wl = 96, 4e-6, 632.8e-9
    x = (np.arange(n) - n / 2) * dx
    ex = np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / (60e-6) ** 2).astype(complex)
    zs = [0.0, 1e-3, 2.5e-3, 5e-3, 1e-2]
    ref = O.propagate3d(O.Field(ex.copy(), dx), zs, method, O.Context(wavelength=wl))
    out = gpu.volume(wos.Field(ex.copy(), dx), zs, method, wos.Context(wavelength=wl))
    assert np.array_equal(out[0, 0], ex)   # z == 0 returns the input unchanged
    for q in range(len(zs)):
        assert rel_l2(out[q], ref[q]) <= tol_case(gpu.precision, method, n, n), q


# ------------------------------------------------------------------ Schell
def test_schell_modes_match_oracle(gpu):
    n, dx, w0, sigc, m = 64, 1e-5, 2e-4, 4e-5, 8
    noise = complex_normal(3, (m, n, n))
    ref = O.schell_realizations(n, dx, w0, sigc, noise)
    got = gpu.schell_modes(n, dx, w0, sigc, noise)
    assert rel_l2(got, ref) <= TOL_FP64_SCHELL   # synthesis runs in FP64 in both precisions


def test_schell_source_coherence_kat(gpu):
    """TestSchellSourceCoherence (coherence_test.go:10-40)."""
    n, dx, w0, sigc, m = 256, 1e-5, 1e-3, 2e-4, 128
    fields = gpu.schell_modes(n, dx, w0, sigc, complex_normal(1, (m, n, n)))
    for dpx in (1, 2, 4, 8, 16):
        a = fields[:, :, : n - dpx]; b = fields[:, :, dpx:]
        num = np.sum(a.real * b.real + a.imag * b.imag)
        got = num / math.sqrt(np.sum(np.abs(a) ** 2) * np.sum(np.abs(b) ** 2))
        assert abs(got - math.exp(-(dpx * dx) ** 2 / (2 * sigc * sigc))) <= 0.03


@pytest.mark.parametrize("method", ["asm", "fraunhofer"])
def test_partially_coherent_matches_oracle(gpu, method):
    n, dx, w0, sigc, m, wl = 64, 1e-5, 2e-4, 4e-5, 12, 632.8e-9
    z = 2e-2 if method == "asm" else 1.0
    noise = complex_normal(5, (m, n, n))
    modes = O.schell_realizations(n, dx, w0, sigc, noise)
    outs = []
    for q in range(m):
        f = O.Field(modes[q].copy(), dx)
        O.propagate(f, z, method, O.Context(wavelength=wl))
        outs.append(f.ex)
    ref = O.average_intensity(np.array(outs))
    got = gpu.partially_coherent(n, dx, w0, sigc, noise, z, method, wos.Context(wavelength=wl))
    assert rel_l2(got, ref) <= max(tol(gpu.precision), TOL_FP64_SCHELL)


# ---------------------------------------------------------------- elements
def _field(n=96, dx=4e-6, pol=False, seed=2):
    rng = np.random.default_rng(seed)
    ex = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    ey = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))) if pol else None
    return ex, ey, dx


@pytest.mark.parametrize("pol", [False, True])
def test_elements_match_oracle(gpu, pol):
    ex, ey, dx = _field(pol=pol)
    wl = 632.8e-9
    cases = [
        ("lens", lambda f, m: m.apply_lens(f, wl, 0.2, 150e-6, 8e-6, -4e-6)),
        ("aperture", lambda f, m: m.apply_aperture_circle(f, 120e-6, 4e-6, 0.0, 0.0)),
        ("aperture_soft", lambda f, m: m.apply_aperture_circle(f, 120e-6, 0.0, 0.0, 10e-6)),
        ("amp_sin", lambda f, m: m.apply_grating(f, "amplitude_sin", 40e-6, 0.7, 0.5, 0, 0.3, 0.2)),
        ("amp_bin", lambda f, m: m.apply_grating(f, "amplitude_binary", 40e-6, 1, 0.3, 0, 0.1, 0)),
        ("phase_sin", lambda f, m: m.apply_grating(f, "phase_sin", 40e-6, 2.0, 0.5, 0, 0.0, 0.4)),
        ("phase_bin", lambda f, m: m.apply_grating(f, "phase_binary", 40e-6, 1.3, 0.5, 0, 0.5, 0)),
        ("blazed", lambda f, m: m.apply_grating(f, "blazed", 40e-6, 1, 0.5, 2.5, 0.2, 0)),
    ]
    for name, fn in cases:
        of = O.Field(ex.copy(), dx, None if ey is None else ey.copy())
        gf = wos.Field(ex.copy(), dx, None if ey is None else ey.copy())
        fn(of, O)
        fn(gf, gpu)
        assert rel_l2(gf.ex, of.ex) <= 1e-13, name   # element arithmetic is FP64 in both precisions
        if pol:
            assert rel_l2(gf.ey, of.ey) <= 1e-13, name
    rng = np.random.default_rng(4)
    phi = rng.uniform(0, 2 * np.pi, ex.shape)
    of = O.Field(ex.copy(), dx); gf = wos.Field(ex.copy(), dx)
    O.apply_phase_mask(of, phi, 0.8); gpu.apply_phase_mask(gf, phi, 0.8)
    assert rel_l2(gf.ex, of.ex) <= 1e-13


def test_element_argument_errors(gpu):
    ex, _, dx = _field(n=16)
    with pytest.raises(wos.WosError):
        gpu.apply_lens(wos.Field(ex, dx), 632.8e-9, 0.0)
    with pytest.raises(wos.WosError):
        gpu.apply_grating(wos.Field(ex, dx), "amplitude_sin", -1.0)


# ---------------------------------------------------------- inverse design
def _design(n=64, seed=0):
    rng = np.random.default_rng(seed)
    phi = rng.uniform(0, 2 * np.pi, (n, n))
    a = np.ones((n, n), complex)
    T = rng.uniform(0, 2, (n, n))
    return a, phi, T


def test_loss_and_gradient_match_oracle(gpu):
    n, dx, wl, z = 64, 4e-6, 633e-9, 2e-3
    a, phi, T = _design(n)
    ctx = O.Context(wavelength=wl)
    lo, go = O.asm_phase_loss_grad(a, phi, T, dx, z, ctx)
    lg, gg = gpu.asm_loss_grad(a, phi, T, dx, z, wos.Context(wavelength=wl))
    t = 1e-11 if gpu.precision == wos.FP64 else 1e-5
    assert abs(lg - lo) / lo <= t
    assert rel_l2(gg, go) <= (1e-11 if gpu.precision == wos.FP64 else 1e-4)
    l2, none = gpu.asm_loss_grad(a, phi, T, dx, z, wos.Context(wavelength=wl), want_grad=False)
    assert none is None and abs(l2 - lg) <= 1e-12 * abs(lg)


def test_gradient_matches_central_differences(gpu):
    """dL/dphi against FP64 central finite differences (h = 1e-6) of the oracle's forward,
    on 64 random pixels, agreeing to 1e-4 (relative to the gradient scale)."""
    n, dx, wl, z = 64, 4e-6, 633e-9, 2e-3
    a, phi, T = _design(n, 1)
    ctx = O.Context(wavelength=wl)
    _, g = gpu.asm_loss_grad(a, phi, T, dx, z, wos.Context(wavelength=wl))
    rng = np.random.default_rng(2)
    scale = np.max(np.abs(g))
    h = 1e-6
    for _ in range(64):
        j, i = rng.integers(0, n, 2)
        p1 = phi.copy(); p1[j, i] += h
        p2 = phi.copy(); p2[j, i] -= h
        l1, _ = O.asm_phase_loss_grad(a, p1, T, dx, z, ctx, want_grad=False)
        l2, _ = O.asm_phase_loss_grad(a, p2, T, dx, z, ctx, want_grad=False)
        fd = (l1 - l2) / (2 * h)
        assert abs(fd - g[j, i]) <= 1e-4 * scale, (j, i, fd, g[j, i])


def test_adjoint_is_the_adjoint(gpu):
    """<A x, y> == <x, A^H y> for the ASM step and its adjoint."""
    n, dx, wl, z = 64, 1e-6, 633e-9, 1e-4
    rng = np.random.default_rng(7)
    xa = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    ya = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    ax = wos.Field(xa.copy(), dx)
    gpu.propagate(ax, z, "asm", wos.Context(wavelength=wl, warnings_enabled=False))
    ahy = wos.Field(ya.copy(), dx)
    gpu.asm_adjoint(ahy, z, wos.Context(wavelength=wl))
    lhs = np.vdot(ya, ax.ex)
    rhs = np.vdot(ahy.ex, xa)
    assert abs(lhs - rhs) / abs(lhs) <= (1e-12 if gpu.precision == wos.FP64 else 1e-5)


def _bpm_dev(g, prec, ex, ey, dx, z, desc, steps, wl, mode):
    """split_step_dev (no diagnostics: the specialised path is eligible) in sweep mode `mode`."""
    import torch
    g.set_fast_path(mode)
    dt = torch.complex128 if prec == wos.FP64 else torch.complex64
    comps = [ex] if ey is None else [ex, ey]
    buf = torch.from_numpy(np.stack(comps)).to(dt).cuda().contiguous()
    torch.cuda.synchronize()
    n = ex.shape[0]
    g.split_step_dev(n, n, dx, len(comps), buf.data_ptr(), z, desc, steps,
                     wos.Context(wavelength=wl, warnings_enabled=False))
    g.synchronize()
    g.set_fast_path(1)
    return buf.cpu().numpy().astype(np.complex128)


@pytest.mark.parametrize("kind", ["uniform", "stratified", "graded", "graded_pol"])
def test_split_step_specialised_matches_general_and_oracle(gpu, kind):
    """The specialised split-step (screen inside the row sweep, slice constants
    applied once, merged half steps as one column step) against the general
    sweeps and the FP64 oracle."""
    n, dx, wl = 128, 0.5e-6, 1.55e-6
    x = (np.arange(n) - n / 2) * dx
    ex = np.exp(-((x[None, :] - 5e-6) ** 2 + x[:, None] ** 2) / (8e-6) ** 2).astype(complex)
    ey = 0.5j * ex if kind == "graded_pol" else None
    if kind == "uniform":
        od, gd = desc_pair(re_bg=1.45, im_bg=1e-5)
        steps, z = 8, 16e-6
    elif kind == "stratified":
        od, gd = desc_pair(re_bg=1.0, im_bg=2e-5, n_layers=2, layer_z=[6e-6, 14e-6], layer_re=[1.5, 1.2],
                           layer_im=[0.0, 1e-4])
        steps, z = 10, 20e-6
    else:
        od, gd = desc_pair(re_bg=1.45, im_bg=1e-5, core_dn=0.01, core_x0=2e-6, core_y0=-3e-6, core_w=25e-6,
                           zmod_amp=0.1, zmod_period=200e-6, zmod_phase=0.3, border_px=16, border_order=2,
                           border_strength=5e-3)
        steps, z = 12, 24e-6
    fast = _bpm_dev(gpu, gpu.precision, ex, ey, dx, z, gd, steps, wl, 1)
    gen = _bpm_dev(gpu, gpu.precision, ex, ey, dx, z, gd, steps, wl, 0)
    of = O.Field(ex.copy(), dx, None if ey is None else ey.copy())
    O.splitstep(of, z, od, steps, O.Context(wavelength=wl))
    t = tol(gpu.precision) * 10
    assert rel_l2(fast[0], of.ex) <= t
    assert rel_l2(fast[0], gen[0]) <= t
    if ey is not None:
        assert rel_l2(fast[1], of.ey) <= t


def test_split_step_specialised_cfg3_scale(gpu):
    """1024^2, 400 slices (the BPM workload): the specialised path against the
    general path in FP64 (both on the GPU; the oracle would take minutes)."""
    n, dx, wl, steps, dz = 1024, 0.5e-6, 1.55e-6, 400, 2e-6
    x = (np.arange(n) - n / 2) * dx
    ex = np.exp(-((x[None, :] - 5e-6) ** 2 + x[:, None] ** 2) / (8e-6) ** 2).astype(complex)
    _, gd = desc_pair(re_bg=1.45, im_bg=1e-5, core_dn=0.01, core_w=25e-6, zmod_amp=0.1, zmod_period=200e-6,
                      border_px=32, border_order=2, border_strength=5e-3)
    fast = _bpm_dev(gpu, gpu.precision, ex, None, dx, steps * dz, gd, steps, wl, 1)
    with wos.GPU(wos.FP64) as g64:
        ref = _bpm_dev(g64, wos.FP64, ex, None, dx, steps * dz, gd, steps, wl, 0)
    err = rel_l2(fast[0], ref[0])
    print("cfg3 rel-L2 vs FP64 general:", err)
    assert err <= (TOL_FP64 if gpu.precision == wos.FP64 else tol_fp32_splitstep(steps))


def test_design_specialised_path_matches_oracle_general_and_fd(gpu):
    """Power-of-two grids take the five-sweep inverse-design path (residual
    and gradient inside the row sweeps): loss and gradient against the FP64
    oracle and the general sweeps, and the gradient against central finite
    differences of the oracle's forward on 16 pixels."""
    n, dx, wl, z = 256, 4e-6, 633e-9, 5e-3
    a, phi, T = _design(n, 3)
    ctx = O.Context(wavelength=wl)
    lo, go = O.asm_phase_loss_grad(a, phi, T, dx, z, ctx)
    lf, gf = gpu.asm_loss_grad(a, phi, T, dx, z, wos.Context(wavelength=wl))
    gpu.set_fast_path(0)
    lg, gg = gpu.asm_loss_grad(a, phi, T, dx, z, wos.Context(wavelength=wl))
    gpu.set_fast_path(1)
    fp64 = gpu.precision == wos.FP64
    assert abs(lf - lo) / lo <= (1e-11 if fp64 else 1e-5)
    assert rel_l2(gf, go) <= (1e-11 if fp64 else 1e-4)
    assert abs(lf - lg) / lg <= (1e-11 if fp64 else 1e-5)
    assert rel_l2(gf, gg) <= (1e-11 if fp64 else 1e-4)
    rng = np.random.default_rng(4)
    scale = np.max(np.abs(gf))
    for _ in range(16):
        j, i = rng.integers(0, n, 2)
        p1 = phi.copy(); p1[j, i] += 1e-6
        p2 = phi.copy(); p2[j, i] -= 1e-6
        l1, _ = O.asm_phase_loss_grad(a, p1, T, dx, z, ctx, want_grad=False)
        l2, _ = O.asm_phase_loss_grad(a, p2, T, dx, z, ctx, want_grad=False)
        assert abs((l1 - l2) / 2e-6 - gf[j, i]) <= 1e-4 * scale


@pytest.mark.parametrize("n", [256, 2048])
def test_design_device_entry_point_matches_host(gpu, n):
    """wos_asm_loss_grad_dev (device arrays, as an optimisation loop keeps
    them) returns the host entry point's loss and gradient."""
    import torch
    dx, wl, z = 4e-6, 633e-9, 0.1 if n == 2048 else 5e-3
    a, phi, T = _design(n, 5)
    lh, gh = gpu.asm_loss_grad(a, phi, T, dx, z, wos.Context(wavelength=wl))
    dt = torch.complex128 if gpu.precision == wos.FP64 else torch.complex64
    ad = torch.from_numpy(a).to(dt).cuda()
    pd = torch.from_numpy(phi).cuda()
    td = torch.from_numpy(T).cuda()
    gd = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ld = gpu.asm_loss_grad_dev(n, n, dx, z, wos.Context(wavelength=wl), ad.data_ptr(), pd.data_ptr(), td.data_ptr(),
                               gd.data_ptr())
    gpu.synchronize()
    fp64 = gpu.precision == wos.FP64
    assert abs(ld - lh) / lh <= (1e-12 if fp64 else 1e-6)
    assert rel_l2(gd.cpu().numpy(), gh) <= (1e-12 if fp64 else 1e-5)
    l0 = gpu.asm_loss_grad_dev(n, n, dx, z, wos.Context(wavelength=wl), ad.data_ptr(), pd.data_ptr(), td.data_ptr())
    assert abs(l0 - ld) <= 1e-12 * abs(ld)


def _general(gpu, fn):
    gpu.set_fast_path(0)
    try:
        return fn()
    finally:
        gpu.set_fast_path(1)


def test_polychromatic_specialised_batch(gpu):
    """256^2 (power of two): the batched specialised sweeps (one shared row
    spectrum, per-wavelength column sweep, intensity accumulated in the row
    sweep) against the oracle and the general sweeps, warnings included."""
    n, dx, z = 256, 2e-6, 2e-2
    x = (np.arange(n) - n / 2) * dx
    g = (np.cos(2 * np.pi * x / 20e-6) >= np.cos(np.pi * 0.5)).astype(float)
    ex = np.tile(g, (n, 1)).astype(complex) * np.exp(-(x[:, None] ** 2) / (150e-6) ** 2)
    wls = np.linspace(400e-9, 700e-9, 9)
    ws = np.linspace(0.5, 1.5, 9)
    oc = O.Context(wavelength=wls[0])
    ref = O.polychromatic(O.Field(ex.copy(), dx), z, wls, ws, "asm", oc)
    gc = wos.Context(wavelength=wls[0])
    out = gpu.polychromatic(wos.Field(ex.copy(), dx), z, wls, ws, "asm", gc)
    gg = wos.Context(wavelength=wls[0])
    gen = _general(gpu, lambda: gpu.polychromatic(wos.Field(ex.copy(), dx), z, wls, ws, "asm", gg))
    assert rel_l2(out, ref) <= tol(gpu.precision)
    assert rel_l2(out, gen) <= tol(gpu.precision)
    check_warnings(gc, oc, gpu.precision == wos.FP64)
    assert gc.warnings.keys() == gg.warnings.keys()


def test_volume_specialised_batch(gpu):
    n, dx, wl = 256, 4e-6, 632.8e-9
    x = (np.arange(n) - n / 2) * dx
    ex = np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / (150e-6) ** 2).astype(complex)
    zs = [0.0, 1e-3, 2.5e-3, 5e-3, 1e-2, 3e-2]
    oc = O.Context(wavelength=wl)
    ref = O.propagate3d(O.Field(ex.copy(), dx), zs, "asm", oc)
    gc = wos.Context(wavelength=wl)
    out = gpu.volume(wos.Field(ex.copy(), dx), zs, "asm", gc)
    gen = _general(gpu, lambda: gpu.volume(wos.Field(ex.copy(), dx), zs, "asm", wos.Context(wavelength=wl)))
    assert np.array_equal(out[0, 0], ex)
    for q in range(len(zs)):
        assert rel_l2(out[q], ref[q]) <= tol(gpu.precision), q
        assert rel_l2(out[q], gen[q]) <= tol(gpu.precision), q
    check_warnings(gc, oc, gpu.precision == wos.FP64)


def test_partially_coherent_fused_synthesis(gpu):
    """Power-of-two grids of 256 points or more without diagnostics: the
    realizations (optics/coherence.go:22-80) are synthesised inside the
    propagation sweeps (the noise times sqrt(S) and the envelope's x factor in
    the first row sweep, its y factor in the column sweep).  Against the
    oracle, and against the path that synthesises them first (which a
    Context with Warnings takes), through the host and the device entry
    points."""
    import torch
    n, dx, w0, sigc, m, wl, z = 256, 1e-5, 6e-4, 5e-5, 7, 632.8e-9, 2e-2
    noise = complex_normal(8, (m, n, n))
    modes = O.schell_realizations(n, dx, w0, sigc, noise)
    outs = []
    for q in range(m):
        f = O.Field(modes[q].copy(), dx)
        O.propagate(f, z, "asm", O.Context(wavelength=wl))
        outs.append(f.ex)
    ref = O.average_intensity(np.array(outs))
    bound = max(tol(gpu.precision), TOL_FP64_SCHELL)
    fused = gpu.partially_coherent(n, dx, w0, sigc, noise, z, "asm", wos.Context(wavelength=wl,
                                                                                   warnings_enabled=False))
    staged = gpu.partially_coherent(n, dx, w0, sigc, noise, z, "asm", wos.Context(wavelength=wl))
    assert rel_l2(fused, ref) <= bound, rel_l2(fused, ref)
    assert rel_l2(staged, ref) <= bound
    assert rel_l2(fused, staged) <= bound
    nd = torch.from_numpy(noise).cuda()
    out = torch.empty((n, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    gpu.partially_coherent_dev(n, dx, w0, sigc, m, nd.data_ptr(), z, wos.Context(wavelength=wl), out.data_ptr())
    gpu.synchronize()
    assert np.array_equal(out.cpu().numpy(), fused)   # the same sweeps on the same noise


def test_partially_coherent_specialised_batch(gpu):
    n, dx, w0, sigc, m, wl, z = 256, 1e-5, 6e-4, 5e-5, 12, 632.8e-9, 2e-2
    noise = complex_normal(6, (m, n, n))
    got = gpu.partially_coherent(n, dx, w0, sigc, noise, z, "asm", wos.Context(wavelength=wl))
    gen = _general(gpu, lambda: gpu.partially_coherent(n, dx, w0, sigc, noise, z, "asm", wos.Context(wavelength=wl)))
    assert rel_l2(got, gen) <= tol(gpu.precision) * 10
