"""At-size parity of every workload of the benchmark table against the FP64
oracle, on the same seeded inputs, through the entry points and launch
configurations that bench.py times:

  cfg1      512^2 plain ASM, lens beam, Evanescent "zero" (complex128 I/O)
  headline  2048^2 ASM, random-phase and lens-beam inputs, autotuned sweeps,
            wos_propagate_batch_dev and wos_propagate_dev
  cfg2      1000 x 1500 asm_shift_pad, two Jones components
  cfg3      1024^2 split-step BPM, 400 slices (the oracle runs all 400)
  cfg4.1    64 wavelengths at 1024^2 (polychromatic)
  cfg4.2    256 Gaussian-Schell modes at 512^2
  cfg4.3    128 planes at 768^2 (volume)
  cfg5      2048^2 phase-mask design: loss and gradient against the oracle
            and against FP64 central differences (h = 1e-6) on 64 pixels
  cfg5.2    3-layer diffractive stack, 200 BPM slices per layer, 2048^2:
            gradient against the FP64 GPU adjoint and central differences

Tolerances (relative L2 against the oracle) come from tests/gpu_util.py:
1e-12 for the FP64 kernels and 1e-5 for the FP32 kernels, with the measured
floors of the carrier-shift, non-power-of-two and Schell cases named there.
Warnings must match the oracle's: the same codes and counts, values within
1e-9 (FP64) or 1e-4 (FP32) relative.  Set WOS_PARITY_LOG to a file path to
append every measured error there as one JSON line.
"""
import importlib
import json
import os

import numpy as np
import pytest

import oracle as O
from gpu_util import TOL_FP32, TOL_FP64, TOL_FP64_SCHELL, rel_l2, tol_case, tol_fp32_splitstep, wos

W = importlib.import_module("tetsuhiro-wos_b200.workloads")

pytestmark = pytest.mark.gpu

PRECS = [pytest.param(wos.FP64, id="fp64"), pytest.param(wos.FP32, id="fp32")]


def pname(prec):
    return "fp64" if prec == wos.FP64 else "fp32"


def record(case, prec, err, bound, **extra):
    """Append one measured error to the WOS_PARITY_LOG file (if set) and check it."""
    path = os.environ.get("WOS_PARITY_LOG")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps(dict(case=case, precision=pname(prec), rel_l2=err, bound=bound, **extra)) + "\n")
    assert err <= bound, (case, pname(prec), err, bound)


def check_warnings(gctx, octx, prec):
    assert set(gctx.warnings) == set(octx.warnings), (gctx.warnings, octx.warnings)
    rt = 1e-9 if prec == wos.FP64 else 1e-4
    for k, (cnt, val) in octx.warnings.items():
        gc, gv = gctx.warnings[k]
        assert gc == cnt, (k, gc, cnt)
        assert abs(gv - val) <= rt * abs(val), (k, gv, val)


def torch_dt(prec):
    import torch
    return torch.complex128 if prec == wos.FP64 else torch.complex64


def to_dev(a, prec):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).to(torch_dt(prec)).cuda().contiguous()
    torch.cuda.synchronize()  # the context's stream does not wait for torch's
    return t


def from_dev(g, t):
    g.synchronize()
    return t.cpu().numpy().astype(np.complex128)


# ------------------------------------------------------------------ cfg1
@pytest.mark.parametrize("prec", PRECS)
def test_cfg1_matches_oracle(prec):
    d = W.cfg1()
    o = O.Field(d["ex"].copy(), d["dx"])
    oc = O.Context(wavelength=d["wl"], evanescent="zero")
    O.propagate(o, d["z"], d["method"], oc)
    with wos.GPU(prec) as g:
        # host complex128 field, Warnings on
        f = wos.Field(d["ex"].copy(), d["dx"])
        gc = wos.Context(wavelength=d["wl"], evanescent="zero")
        diag = g.propagate(f, d["z"], d["method"], gc)
        assert diag.wrap_checked == 1
        record("cfg1 host", prec, rel_l2(f.ex, o.ex), TOL_FP64 if prec == wos.FP64 else TOL_FP32)
        check_warnings(gc, oc, prec)
        # device-resident, as the benchmark times it (Warnings off)
        buf = to_dev(d["ex"][None], prec)
        g.propagate_dev(512, 512, d["dx"], 1, buf.data_ptr(), buf.data_ptr(), d["z"], d["method"],
                        wos.Context(wavelength=d["wl"], evanescent="zero", warnings_enabled=False))
        record("cfg1 device", prec, rel_l2(from_dev(g, buf)[0], o.ex), TOL_FP64 if prec == wos.FP64 else TOL_FP32)


# ------------------------------------------------------------------ headline
@pytest.fixture(scope="module")
def headline_ref():
    h = W.HEADLINE
    out = {}
    for name, ex in (("random_phase", W.random_phase(h["n"])), ("lens", W.lens_beam(h["n"], h["dx"], h["wl"]))):
        o = O.Field(ex.copy(), h["dx"])
        oc = O.Context(wavelength=h["wl"])
        O.propagate(o, h["z"], "asm", oc)
        out[name] = (ex, o.ex, oc)
    return out


@pytest.mark.parametrize("prec", PRECS)
def test_headline_2048_matches_oracle(prec, headline_ref):
    """The benchmark's own path at 2048^2: the autotuned launch configuration,
    a two-field wos_propagate_batch_dev (the fields run on two streams), one
    wos_propagate_dev per field, and the host call with Warnings on."""
    h = W.HEADLINE
    n = h["n"]
    bound = TOL_FP64 if prec == wos.FP64 else TOL_FP32
    names = list(headline_ref)
    with wos.GPU(prec) as g:
        g.autotune(n, n)
        quiet = wos.Context(wavelength=h["wl"], warnings_enabled=False)
        bufs = [to_dev(headline_ref[k][0], prec) for k in names]
        ptrs = [b.data_ptr() for b in bufs]
        g.propagate_batch_dev(n, n, h["dx"], 1, ptrs, ptrs, h["z"], "asm", quiet)
        for k, b in zip(names, bufs):
            record(f"headline batch_dev {k}", prec, rel_l2(from_dev(g, b), headline_ref[k][1]), bound)
        for k in names:
            b = to_dev(headline_ref[k][0], prec)
            g.propagate_dev(n, n, h["dx"], 1, b.data_ptr(), b.data_ptr(), h["z"], "asm", quiet)
            record(f"headline dev {k}", prec, rel_l2(from_dev(g, b), headline_ref[k][1]), bound)
        for k in names:
            f = wos.Field(headline_ref[k][0].copy(), h["dx"])
            gc = wos.Context(wavelength=h["wl"])
            diag = g.propagate(f, h["z"], "asm", gc)
            assert diag.wrap_checked == 1
            record(f"headline host {k}", prec, rel_l2(f.ex, headline_ref[k][1]), bound)
            check_warnings(gc, headline_ref[k][2], prec)


# ------------------------------------------------------------------ cfg2
@pytest.mark.parametrize("prec", PRECS)
def test_cfg2_matches_oracle(prec):
    d = W.cfg2()
    o = O.Field(d["ex"].copy(), d["dx"], d["ey"].copy())
    oc = O.Context(wavelength=d["wl"])
    O.propagate(o, d["z"], d["method"], oc)
    ny, nx = d["ex"].shape
    bound = tol_case(prec, d["method"], ny, nx)
    with wos.GPU(prec) as g:
        f = wos.Field(d["ex"].copy(), d["dx"], d["ey"].copy())
        gc = wos.Context(wavelength=d["wl"])
        diag = g.propagate(f, d["z"], d["method"], gc)
        assert diag.carrier_applied == 1
        record("cfg2 host ex", prec, rel_l2(f.ex, o.ex), bound)
        record("cfg2 host ey", prec, rel_l2(f.ey, o.ey), bound)
        check_warnings(gc, oc, prec)
        buf = to_dev(np.stack([d["ex"], d["ey"]]), prec)
        g.propagate_dev(ny, nx, d["dx"], 2, buf.data_ptr(), buf.data_ptr(), d["z"], d["method"],
                        wos.Context(wavelength=d["wl"], warnings_enabled=False))
        r = from_dev(g, buf)
        record("cfg2 device", prec, rel_l2(r, np.stack([o.ex, o.ey])), bound)


# ------------------------------------------------------------------ cfg3
@pytest.fixture(scope="module")
def cfg3_ref():
    d = W.cfg3()
    o = O.Field(d["ex"].copy(), d["dx"])
    O.splitstep(o, d["z"], W.index_desc(O.IndexDesc, d["desc"]), d["steps"], O.Context(wavelength=d["wl"]))
    return d, o.ex


@pytest.mark.parametrize("prec", PRECS)
def test_cfg3_bpm_400_slices_matches_oracle(prec, cfg3_ref):
    """The whole 400-slice run against the oracle's 400 slices."""
    d, ref = cfg3_ref
    n = d["ex"].shape[0]
    desc = W.index_desc(wos.IndexDesc, d["desc"])
    with wos.GPU(prec) as g:
        buf = to_dev(d["ex"], prec)
        g.split_step_dev(n, n, d["dx"], 1, buf.data_ptr(), d["z"], desc, d["steps"],
                         wos.Context(wavelength=d["wl"], warnings_enabled=False))
        bound = TOL_FP64 if prec == wos.FP64 else tol_fp32_splitstep(d["steps"])
        record("cfg3 device", prec, rel_l2(from_dev(g, buf), ref), bound)
        # the host entry point with the reference's default Context (Warnings
        # nil); with Warnings on, the per-half-step power sums take the general
        # sweeps, which the small-grid split-step tests check
        f = wos.Field(d["ex"].copy(), d["dx"])
        g.split_step(f, d["z"], desc, d["steps"], wos.Context(wavelength=d["wl"], warnings_enabled=False))
        record("cfg3 host", prec, rel_l2(f.ex, ref), bound)


# ------------------------------------------------------------------ cfg4
@pytest.mark.parametrize("prec", PRECS)
def test_cfg4_1_polychromatic_matches_oracle(prec):
    d = W.cfg4_1()
    oc = O.Context(wavelength=d["wls"][0])
    ref = O.polychromatic(O.Field(d["ex"].copy(), d["dx"]), d["z"], d["wls"], d["weights"], "asm", oc)
    with wos.GPU(prec) as g:
        gc = wos.Context(wavelength=d["wls"][0])
        got = g.polychromatic(wos.Field(d["ex"].copy(), d["dx"]), d["z"], d["wls"], d["weights"], "asm", gc)
    record("cfg4.1", prec, rel_l2(got, ref), TOL_FP64 if prec == wos.FP64 else TOL_FP32)
    check_warnings(gc, oc, prec)
    # the device-resident form on a device field
    import torch
    n = d["ex"].shape[0]
    with wos.GPU(prec) as g:
        fd = to_dev(d["ex"][None], prec)
        out = torch.empty((n, n), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        g.polychromatic_dev(n, n, d["dx"], 1, fd.data_ptr(), d["z"], d["wls"], d["weights"],
                            wos.Context(wavelength=d["wls"][0]), out.data_ptr())
        g.synchronize()
        record("cfg4.1 device", prec, rel_l2(out.cpu().numpy(), ref), TOL_FP64 if prec == wos.FP64 else TOL_FP32)


@pytest.fixture(scope="module")
def cfg4_2_ref():
    d = W.cfg4_2()
    modes = O.schell_realizations(d["n"], d["dx"], d["width"], d["coherence"], d["noise"])
    for k in range(modes.shape[0]):
        f = O.Field(modes[k], d["dx"])
        O.propagate(f, d["z"], "asm", O.Context(wavelength=d["wl"], warnings_enabled=False))
        modes[k] = f.ex
    return d, O.average_intensity(modes)


@pytest.mark.parametrize("prec", PRECS)
def test_cfg4_2_partially_coherent_matches_oracle(prec, cfg4_2_ref):
    d, ref = cfg4_2_ref
    with wos.GPU(prec) as g:
        got = g.partially_coherent(d["n"], d["dx"], d["width"], d["coherence"], d["noise"], d["z"], "asm",
                                   wos.Context(wavelength=d["wl"], warnings_enabled=False))
    record("cfg4.2", prec, rel_l2(got, ref), TOL_FP64_SCHELL if prec == wos.FP64 else TOL_FP32)
    import torch
    with wos.GPU(prec) as g:
        nd = torch.from_numpy(d["noise"]).cuda()
        out = torch.empty((d["n"], d["n"]), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        g.partially_coherent_dev(d["n"], d["dx"], d["width"], d["coherence"], d["noise"].shape[0], nd.data_ptr(),
                                 d["z"], wos.Context(wavelength=d["wl"], warnings_enabled=False), out.data_ptr())
        g.synchronize()
        record("cfg4.2 device", prec, rel_l2(out.cpu().numpy(), ref), TOL_FP64_SCHELL if prec == wos.FP64 else TOL_FP32)


@pytest.fixture(scope="module")
def cfg4_3_ref():
    d = W.cfg4_3()
    oc = O.Context(wavelength=d["wl"])
    ref = O.propagate3d(O.Field(d["ex"].copy(), d["dx"]), d["zs"], "asm", oc)
    return d, ref, oc


@pytest.mark.parametrize("prec", PRECS)
def test_cfg4_3_volume_matches_oracle(prec, cfg4_3_ref):
    d, ref, oc = cfg4_3_ref
    n = d["ex"].shape[0]
    with wos.GPU(prec) as g:
        gc = wos.Context(wavelength=d["wl"])
        got = g.volume(wos.Field(d["ex"].copy(), d["dx"]), d["zs"], "asm", gc)
    assert rel_l2(got[0, 0], d["ex"]) <= (0.0 if prec == wos.FP64 else 1e-7)  # z = 0 returns the input
    record("cfg4.3", prec, rel_l2(got, ref), tol_case(prec, "asm", n, n))
    check_warnings(gc, oc, prec)
    del got
    import torch
    with wos.GPU(prec) as g:
        fd = to_dev(d["ex"][None], prec)
        out = torch.empty((d["zs"].size, 1, n, n), dtype=torch_dt(prec), device="cuda")
        torch.cuda.synchronize()
        g.volume_dev(n, n, d["dx"], 1, fd.data_ptr(), d["zs"], wos.Context(wavelength=d["wl"]), out.data_ptr())
        g.synchronize()
        dev = out.cpu().numpy().astype(np.complex128)
    record("cfg4.3 device", prec, rel_l2(dev, ref), tol_case(prec, "asm", n, n))


@pytest.mark.parametrize("prec", PRECS)
def test_cfg4_device_batches_replay_from_one_graph(prec):
    """The three device-resident batches recorded in one CUDA graph: a replay
    reproduces the direct calls exactly (fewer units than the benchmark, same
    grids)."""
    import torch
    d1, d2, d3 = W.cfg4_1(), W.cfg4_2(16), W.cfg4_3(16)
    n1, n2, n3 = d1["ex"].shape[0], d2["n"], d3["ex"].shape[0]
    with wos.GPU(prec) as g:
        f1 = to_dev(d1["ex"][None], prec)
        f3 = to_dev(d3["ex"][None], prec)
        nz = torch.from_numpy(d2["noise"]).cuda()
        o1 = torch.empty((n1, n1), dtype=torch.float64, device="cuda")
        o2 = torch.empty((n2, n2), dtype=torch.float64, device="cuda")
        o3 = torch.empty((d3["zs"].size, 1, n3, n3), dtype=torch_dt(prec), device="cuda")
        torch.cuda.synchronize()

        def run():
            g.polychromatic_dev(n1, n1, d1["dx"], 1, f1.data_ptr(), d1["z"], d1["wls"], d1["weights"],
                                wos.Context(wavelength=d1["wls"][0]), o1.data_ptr())
            g.partially_coherent_dev(n2, d2["dx"], d2["width"], d2["coherence"], 16, nz.data_ptr(), d2["z"],
                                     wos.Context(wavelength=d2["wl"]), o2.data_ptr())
            g.volume_dev(n3, n3, d3["dx"], 1, f3.data_ptr(), d3["zs"], wos.Context(wavelength=d3["wl"]),
                         o3.data_ptr())
        run()
        g.synchronize()
        direct = [o1.cpu().numpy(), o2.cpu().numpy(), o3.cpu().numpy()]
        for o in (o1, o2, o3):
            o.zero_()
        torch.cuda.synchronize()
        g.graph_capture_begin()
        run()
        gr = g.graph_capture_end()
        gr.launch()
        g.synchronize()
        replay = [o1.cpu().numpy(), o2.cpu().numpy(), o3.cpu().numpy()]
        gr.close()
    for a, b in zip(direct, replay):
        assert np.array_equal(a, b)


# ------------------------------------------------------------------ cfg5
def _fd_pixels(rng, n, count=64):
    return [tuple(int(v) for v in rng.integers(0, n, 2)) for _ in range(count)]


def _loss_difference(up, um, target):
    """L(+) - L(-) for L = sum (|u|^2 - T)^2, formed pixel by pixel as
    (I+ - I-)(I+ + I- - 2T): the loss itself is ~1e7 at 2048^2, so two rounded
    losses would differ by their rounding (~1e-9) more than by h g (~1e-6)."""
    ip = up.real ** 2 + up.imag ** 2
    im = um.real ** 2 + um.imag ** 2
    return float(np.sum((ip - im) * (ip + im - 2 * target)))


@pytest.fixture(scope="module")
def cfg5_ref():
    d = W.cfg5()
    ctx = O.Context(wavelength=d["wl"], warnings_enabled=False)
    loss, grad = O.asm_phase_loss_grad(d["a"], d["phi"], d["target"], d["dx"], d["z"], ctx)
    rng = np.random.default_rng(2)
    h = 1e-6
    fd = []
    for (j, i) in _fd_pixels(rng, d["phi"].shape[0]):
        us = []
        for s in (h, -h):
            p = d["phi"].copy()
            p[j, i] += s
            f = O.Field(d["a"] * np.exp(1j * p), d["dx"])
            O.propagate(f, d["z"], "asm", O.Context(wavelength=d["wl"], warnings_enabled=False))
            us.append(f.ex)
        fd.append(((j, i), _loss_difference(us[0], us[1], d["target"]) / (2 * h)))
    return d, loss, grad, fd


@pytest.mark.parametrize("prec", PRECS)
def test_cfg5_design_gradient_matches_oracle_and_fd(prec, cfg5_ref):
    """wos_asm_loss_grad_dev (the benchmark's call) at 2048^2: loss and
    gradient against the oracle's FP64 adjoint, and the gradient against FP64
    central differences (h = 1e-6) of the oracle's forward on 64 pixels."""
    import torch
    d, loss_o, grad_o, fd = cfg5_ref
    n = d["phi"].shape[0]
    with wos.GPU(prec) as g:
        ad = to_dev(d["a"], prec)
        pd = torch.from_numpy(d["phi"]).cuda()
        td = torch.from_numpy(d["target"]).cuda()
        gd = torch.empty((n, n), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        loss = g.asm_loss_grad_dev(n, n, d["dx"], d["z"], wos.Context(wavelength=d["wl"]), ad.data_ptr(),
                                   pd.data_ptr(), td.data_ptr(), gd.data_ptr())
        g.synchronize()
        grad = gd.cpu().numpy()
    fp64 = prec == wos.FP64
    record("cfg5 loss", prec, abs(loss - loss_o) / loss_o, 1e-12 if fp64 else 1e-5)
    record("cfg5 grad vs oracle adjoint", prec, rel_l2(grad, grad_o), 1e-12 if fp64 else 1e-4)
    fdv = np.array([v for _, v in fd])
    gv = np.array([grad[p] for p, _ in fd])
    record("cfg5 grad vs FD (64 px)", prec, float(np.linalg.norm(gv - fdv) / np.linalg.norm(fdv)), 1e-4,
           max_abs_over_max=float(np.max(np.abs(gv - fdv)) / np.max(np.abs(fdv))))


@pytest.fixture(scope="module")
def cfg5_2_ref():
    """The FP64 GPU adjoint of the stack, and FP64 central differences of the
    stack's forward composed from the FP64 split-step (mask multiply, then
    wos_splitstep_dev per layer) on 64 pixels spread over the three masks."""
    import torch
    d = W.cfg5_2()
    nl, n = d["phis"].shape[0], d["phis"].shape[1]
    desc = W.index_desc(wos.IndexDesc, d["desc"])
    ctx = wos.Context(wavelength=d["wl"], warnings_enabled=False)
    with wos.GPU(wos.FP64) as g:
        ad = to_dev(d["a"], wos.FP64)
        pd = torch.from_numpy(d["phis"]).cuda()
        td = torch.from_numpy(d["target"]).cuda()
        gd = torch.empty((nl, n, n), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        loss = g.bpm_stack_loss_grad_dev(ad.data_ptr(), pd.data_ptr(), td.data_ptr(), gd.data_ptr(), nl, n, n,
                                         d["dx"], d["zseg"], d["steps"], desc, ctx)
        g.synchronize()
        grads = gd.cpu().numpy()

        def forward(phis):
            u = torch.from_numpy(d["a"]).cuda()
            for l in range(nl):
                u = u * torch.exp(1j * torch.from_numpy(phis[l]).cuda())
                u = u.contiguous()
                torch.cuda.synchronize()
                g.split_step_dev(n, n, d["dx"], 1, u.data_ptr(), d["zseg"], desc, d["steps"], ctx)
                g.synchronize()
            return u.cpu().numpy()

        rng = np.random.default_rng(2)
        h = 1e-6
        fd = []
        for k in range(64):
            l = k % nl
            j, i = (int(v) for v in rng.integers(0, n, 2))
            us = []
            for s in (h, -h):
                p = d["phis"].copy()
                p[l, j, i] += s
                us.append(forward(p))
            fd.append(((l, j, i), _loss_difference(us[0], us[1], d["target"]) / (2 * h)))
    return d, loss, grads, fd


@pytest.mark.parametrize("prec", PRECS)
def test_cfg5_2_stack_gradient_matches_fp64_adjoint_and_fd(prec, cfg5_2_ref):
    import torch
    d, loss64, grads64, fd = cfg5_2_ref
    nl, n = d["phis"].shape[0], d["phis"].shape[1]
    with wos.GPU(prec) as g:
        ad = to_dev(d["a"], prec)
        pd = torch.from_numpy(d["phis"]).cuda()
        td = torch.from_numpy(d["target"]).cuda()
        gd = torch.empty((nl, n, n), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        loss = g.bpm_stack_loss_grad_dev(ad.data_ptr(), pd.data_ptr(), td.data_ptr(), gd.data_ptr(), nl, n, n,
                                         d["dx"], d["zseg"], d["steps"], W.index_desc(wos.IndexDesc, d["desc"]),
                                         wos.Context(wavelength=d["wl"], warnings_enabled=False))
        g.synchronize()
        grads = gd.cpu().numpy()
    fp64 = prec == wos.FP64
    if not fp64:
        # 600 slices (field error ~2e-5); the loss (|u|^2 - T)^2 amplifies it
        # about threefold (measured 6.2e-5); held to the gradient's 1e-4
        record("cfg5.2 loss vs FP64 GPU", prec, abs(loss - loss64) / loss64, 1e-4)
        record("cfg5.2 grads vs FP64 GPU adjoint", prec, rel_l2(grads, grads64), 1e-4)
    fdv = np.array([v for _, v in fd])
    gv = np.array([grads[p] for p, _ in fd])
    record("cfg5.2 grads vs FD (64 px)", prec, float(np.linalg.norm(gv - fdv) / np.linalg.norm(fdv)), 1e-4,
           max_abs_over_max=float(np.max(np.abs(gv - fdv)) / np.max(np.abs(fdv))))
