"""CUDA graphs of device-resident calls (wos_graph_capture_begin / _end,
wos_graph_launch): a replay must give the results of the captured calls run
directly (bit for bit: the same kernels on the same buffers), including the
forked streams of a device batch, branches on other contexts
(wos_graph_capture_fork / _join) and in-place split-step runs replayed
repeatedly; a call that needs a synchronisation inside a capture fails cleanly
and leaves the context usable."""
import numpy as np
import pytest

from gpu_util import wos

pytestmark = pytest.mark.gpu

PRECS = [pytest.param(wos.FP64, id="fp64"), pytest.param(wos.FP32, id="fp32")]


@pytest.fixture(scope="module", params=PRECS)
def gpu(request):
    g = wos.GPU(request.param)
    yield g
    g.close()


def _dt(gpu):
    import torch
    return torch.complex128 if gpu.precision == wos.FP64 else torch.complex64


def _fields(gpu, k, n, seed=1):
    import torch
    rng = np.random.default_rng(seed)
    return [torch.from_numpy(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))).to(_dt(gpu)).cuda()
            for _ in range(k)]


CTX = dict(wavelength=632.8e-9, warnings_enabled=False)


def test_graph_keeps_its_tables_while_other_calls_evict(gpu):
    """A graph reads the transfer-function table and the parameter lists of its
    capture even after later direct calls with many other distances and
    wavelength lists have cycled the context's caches."""
    import torch
    n, dx, z = 512, 2e-6, 5e-3
    (x,) = _fields(gpu, 1, n, seed=3)
    y = torch.empty_like(x)
    want = torch.empty_like(x)
    wls = np.linspace(500e-9, 600e-9, 3)
    pw = torch.empty((n, n), dtype=torch.float64, device="cuda")
    pw_want = torch.empty_like(pw)
    torch.cuda.synchronize()

    def calls(out, pout):
        gpu.propagate_dev(n, n, dx, 1, x.data_ptr(), out.data_ptr(), z, "asm", wos.Context(**CTX))
        gpu.polychromatic_dev(n, n, dx, 1, x.data_ptr(), z, wls, np.ones(3), wos.Context(**CTX), pout.data_ptr())

    calls(want, pw_want)
    gpu.synchronize()
    gpu.graph_capture_begin()
    calls(y, pw)
    g = gpu.graph_capture_end()
    scratch = torch.empty_like(x)
    sp = torch.empty_like(pw)
    for q in range(12):  # other distances and wavelength lists, more than either cache holds
        gpu.propagate_dev(n, n, dx, 1, x.data_ptr(), scratch.data_ptr(), z * (1.1 + 0.1 * q), "asm",
                          wos.Context(**CTX))
        gpu.polychromatic_dev(n, n, dx, 1, x.data_ptr(), z, wls * (1.01 + 0.01 * q), np.ones(3),
                              wos.Context(**CTX), sp.data_ptr())
    gpu.synchronize()
    y.zero_()
    pw.zero_()
    torch.cuda.synchronize()
    g.launch()
    gpu.synchronize()
    assert torch.equal(y, want)
    assert torch.equal(pw, pw_want)
    g.close()


def test_graph_replays_single_calls(gpu):
    import torch
    n, dx, z = 512, 2e-6, 5e-3
    ins = _fields(gpu, 3, n)
    outs = [torch.empty_like(t) for t in ins]
    want = [torch.empty_like(t) for t in ins]
    torch.cuda.synchronize()
    for i, w in zip(ins, want):  # direct calls (also the warm-up of the capture)
        gpu.propagate_dev(n, n, dx, 1, i.data_ptr(), w.data_ptr(), z, "asm", wos.Context(**CTX))
    gpu.synchronize()
    gpu.graph_capture_begin()
    for i, o in zip(ins, outs):
        gpu.propagate_dev(n, n, dx, 1, i.data_ptr(), o.data_ptr(), z, "asm", wos.Context(**CTX))
    g = gpu.graph_capture_end()
    for _ in range(2):
        for o in outs:
            o.zero_()
        torch.cuda.synchronize()
        g.launch()
        gpu.synchronize()
        for o, w in zip(outs, want):
            assert torch.equal(o, w)
    g.close()


def test_graph_replays_a_device_batch_on_forked_streams(gpu):
    import torch
    n, dx, z = 1024, 2e-6, 2e-2
    ins = _fields(gpu, 4, n, 2)
    outs = [torch.empty_like(t) for t in ins]
    torch.cuda.synchronize()
    gpu.propagate_batch_dev(n, n, dx, 1, [t.data_ptr() for t in ins], [t.data_ptr() for t in outs], z, "asm",
                            wos.Context(**CTX))
    gpu.synchronize()
    want = [o.clone() for o in outs]
    gpu.graph_capture_begin()
    gpu.propagate_batch_dev(n, n, dx, 1, [t.data_ptr() for t in ins], [t.data_ptr() for t in outs], z, "asm",
                            wos.Context(**CTX))
    g = gpu.graph_capture_end()
    for o in outs:
        o.zero_()
    torch.cuda.synchronize()
    g.launch()
    gpu.synchronize()
    for o, w in zip(outs, want):
        assert torch.equal(o, w)
    g.close()


def test_graph_replays_split_step_in_place(gpu):
    """Each replay advances the field by one captured BPM run, like a direct call."""
    import torch
    n, dx = 256, 0.5e-6
    d = wos.IndexDesc()
    d.re_bg, d.core_dn, d.core_w, d.border_px, d.border_order, d.border_strength = 1.45, 0.01, 20e-6, 8, 2, 5e-3
    ctx = dict(wavelength=1.55e-6, warnings_enabled=False)
    a = _fields(gpu, 1, n, 3)[0]
    b = a.clone()
    torch.cuda.synchronize()
    gpu.split_step_dev(n, n, dx, 1, a.data_ptr(), 20e-6, d, 10, wos.Context(**ctx))  # warm-up, direct
    gpu.split_step_dev(n, n, dx, 1, a.data_ptr(), 20e-6, d, 10, wos.Context(**ctx))
    gpu.synchronize()
    gpu.graph_capture_begin()
    gpu.split_step_dev(n, n, dx, 1, b.data_ptr(), 20e-6, d, 10, wos.Context(**ctx))
    g = gpu.graph_capture_end()
    torch.cuda.synchronize()
    g.launch()
    g.launch()
    gpu.synchronize()
    assert torch.equal(a, b)
    g.close()


def test_graph_capture_of_a_synchronising_call_fails_cleanly(gpu):
    import torch
    n, dx, z = 256, 2e-6, 1e-3
    x = _fields(gpu, 1, n, 4)[0]
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    gpu.graph_capture_begin()
    with pytest.raises(wos.WosError):
        # the carrier-shift methods read the spectral centroid back to the host
        gpu.propagate_dev(n, n, dx, 1, x.data_ptr(), y.data_ptr(), z, "asm_shift", wos.Context(**CTX))
    with pytest.raises(wos.WosError):
        gpu.graph_capture_end()
    gpu.propagate_dev(n, n, dx, 1, x.data_ptr(), y.data_ptr(), z, "asm", wos.Context(**CTX))
    gpu.synchronize()
    assert torch.isfinite(torch.view_as_real(y)).all()


def test_graph_branches_of_other_contexts(gpu):
    """wos_graph_capture_fork / _join: the calls of two more contexts, recorded
    as concurrent branches of one capture, replay with the results of the
    direct calls (bit for bit); misuse fails without breaking the capture."""
    import torch
    n, dx = 512, 2e-6
    other = [wos.GPU(gpu.precision) for _ in range(2)]
    try:
        ins = _fields(gpu, 3, n, 7)
        outs = [torch.empty_like(t) for t in ins]
        wls = np.linspace(500e-9, 600e-9, 3)
        pw = torch.empty((n, n), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()

        def calls():
            gpu.propagate_dev(n, n, dx, 1, ins[0].data_ptr(), outs[0].data_ptr(), 5e-3, "asm", wos.Context(**CTX))
            other[0].propagate_batch_dev(n, n, dx, 1, [ins[1].data_ptr(), ins[2].data_ptr()],
                                         [outs[1].data_ptr(), outs[2].data_ptr()], 2e-3, "asm", wos.Context(**CTX))
            other[1].polychromatic_dev(n, n, dx, 1, ins[0].data_ptr(), 1e-2, wls, np.ones(3), wos.Context(**CTX),
                                       pw.data_ptr())

        calls()  # direct, also the warm-up of the capture
        for g in [gpu] + other:
            g.synchronize()
        want = [o.clone() for o in outs] + [pw.clone()]
        with pytest.raises(wos.WosError):
            gpu.graph_capture_fork(other[0])  # ctx is not capturing
        gpu.graph_capture_begin()
        gpu.graph_capture_fork(other[0])
        gpu.graph_capture_fork(other[1])
        with pytest.raises(wos.WosError):
            gpu.graph_capture_fork(other[0])  # already a branch
        calls()
        with pytest.raises(wos.WosError):
            gpu.graph_capture_end()  # branches still open
        gpu.graph_capture_join(other[0])
        gpu.graph_capture_join(other[1])
        with pytest.raises(wos.WosError):
            gpu.graph_capture_join(other[1])  # already joined
        g = gpu.graph_capture_end()
        for _ in range(2):
            for o in outs:
                o.zero_()
            pw.zero_()
            torch.cuda.synchronize()
            g.launch()
            gpu.synchronize()
            for o, w in zip(outs + [pw], want):
                assert torch.equal(o, w)
        g.close()
        # the branches' contexts are usable on their own again
        other[0].propagate_dev(n, n, dx, 1, ins[1].data_ptr(), outs[1].data_ptr(), 2e-3, "asm", wos.Context(**CTX))
        other[0].synchronize()
        assert torch.equal(outs[1], want[1])
    finally:
        for g in other:
            g.close()


def test_graph_branch_destroyed_mid_capture(gpu):
    """A context destroyed while it is a branch of a capture: the owner's
    capture then fails at its end and the owner works on; an owner destroyed
    with a branch open ends its capture, and the branch works on."""
    import torch
    n, dx, z = 256, 2e-6, 1e-3
    x = _fields(gpu, 1, n, 9)[0]
    y, want = torch.empty_like(x), torch.empty_like(x)
    torch.cuda.synchronize()
    gpu.propagate_dev(n, n, dx, 1, x.data_ptr(), want.data_ptr(), z, "asm", wos.Context(**CTX))
    gpu.synchronize()
    b = wos.GPU(gpu.precision)
    b.propagate_dev(n, n, dx, 1, x.data_ptr(), y.data_ptr(), z, "asm", wos.Context(**CTX))
    b.synchronize()
    gpu.graph_capture_begin()
    gpu.graph_capture_fork(b)
    b.propagate_dev(n, n, dx, 1, x.data_ptr(), y.data_ptr(), z, "asm", wos.Context(**CTX))
    b.close()
    with pytest.raises(wos.WosError):
        gpu.graph_capture_end()
    y.zero_()
    torch.cuda.synchronize()
    gpu.propagate_dev(n, n, dx, 1, x.data_ptr(), y.data_ptr(), z, "asm", wos.Context(**CTX))
    gpu.synchronize()
    assert torch.equal(y, want)

    owner, b = wos.GPU(gpu.precision), wos.GPU(gpu.precision)
    owner.propagate_dev(n, n, dx, 1, x.data_ptr(), y.data_ptr(), z, "asm", wos.Context(**CTX))
    owner.synchronize()
    owner.graph_capture_begin()
    owner.graph_capture_fork(b)
    owner.close()
    y.zero_()
    torch.cuda.synchronize()
    b.propagate_dev(n, n, dx, 1, x.data_ptr(), y.data_ptr(), z, "asm", wos.Context(**CTX))
    b.synchronize()
    assert torch.equal(y, want)
    b.close()
