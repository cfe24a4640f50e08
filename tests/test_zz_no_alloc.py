"""The zero-padded ASM entry point that allocates no device memory.

Some callers cannot call cudaMalloc: processes that reserve every byte of a
GPU up front behind their own allocator, or pipelines that cannot afford the
device-wide synchronisation of cudaFree.  wos_asm_pad_c64_noalloc serves them
from file-scope device arrays instead of a context workspace.  These checks
call it through the C ABI and compare it with the regular asm_pad entry point
(same tolerance as the other FP32 parity tests), on two calls in a row with
different inputs, and with the FP64 oracle forward and backward (with and
without Tikhonov regularisation), at zero distance, in place, and on the
smallest and non-square grids; sizes beyond its static workspace are
rejected.  The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from gpu_util import TOL_FP32, rel_l2, wos

pytestmark = pytest.mark.gpu


def _noalloc(in_ptr, out_ptr, ny, nx, dx, z, wl, stream, ctx=None):
    cc = (ctx or wos.Context(wavelength=wl, warnings_enabled=False)).c()
    return wos.lib().wos_asm_pad_c64_noalloc(C.c_void_p(in_ptr), C.c_void_p(out_ptr), ny, nx, dx, z,
                                              C.byref(cc), C.c_void_p(stream))


def _field(ny, nx, dx, seed):
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) - nx / 2) * dx
    y = (np.arange(ny) - ny / 2) * dx
    env = np.exp(-(x[None, :] ** 2 + y[:, None] ** 2) / (0.3 * max(nx, ny) * dx) ** 2)
    return (env * np.exp(1j * rng.uniform(0, 2 * np.pi, (ny, nx)))).astype(np.complex64)


def _run_noalloc(ex, dx, z, ctx, inplace=False):
    import torch
    ny, nx = ex.shape
    src = torch.from_numpy(ex).cuda()
    out = src if inplace else torch.empty_like(src)
    torch.cuda.synchronize()
    rc = _noalloc(src.data_ptr(), out.data_ptr(), ny, nx, dx, z, ctx.wavelength, 0, ctx)
    assert rc == 0, wos.lib().wos_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy().astype(np.complex128)


def test_noalloc_asm_pad_matches_context_entry_point():
    import torch
    ny, nx, dx, wl, z = 256, 512, 2e-6, 632.8e-9, 4e-3
    rng = np.random.default_rng(11)
    stream = torch.cuda.Stream()
    with wos.GPU(wos.FP32) as g:
        g.set_stream(stream.cuda_stream)
        for call in range(2):   # two calls in a row share the static workspace
            x = (np.arange(nx) - nx / 2) * dx
            y = (np.arange(ny) - ny / 2) * dx
            env = np.exp(-(x[None, :] ** 2 + y[:, None] ** 2) / (150e-6 + 50e-6 * call) ** 2)
            ex = (env * np.exp(1j * rng.uniform(0, 2 * np.pi, (ny, nx)))).astype(np.complex64)
            with torch.cuda.stream(stream):
                src = torch.from_numpy(ex).cuda()
                out = torch.empty_like(src)
                ref = src.clone()
            torch.cuda.synchronize()
            rc = _noalloc(src.data_ptr(), out.data_ptr(), ny, nx, dx, z, wl, stream.cuda_stream)
            assert rc == 0, wos.lib().wos_last_error()
            g.propagate_dev(ny, nx, dx, 1, ref.data_ptr(), ref.data_ptr(), z, "asm_pad",
                            wos.Context(wavelength=wl, warnings_enabled=False))
            torch.cuda.synchronize()
            a = out.cpu().numpy().astype(np.complex128)
            b = ref.cpu().numpy().astype(np.complex128)
            assert np.all(np.isfinite(a))
            assert rel_l2(a, b) <= TOL_FP32, (call, rel_l2(a, b))


def test_noalloc_rejects_sizes_beyond_its_workspace():
    import torch
    t = torch.zeros((4, 4), dtype=torch.complex64, device="cuda")
    for ny, nx in ((2048, 8), (8, 2048), (100, 128)):
        rc = _noalloc(t.data_ptr(), t.data_ptr(), ny, nx, 1e-6, 1e-3, 5e-7, 0)
        assert rc == 2   # WOS_UNSUPPORTED_SIZE
        assert b"1024" in wos.lib().wos_last_error() or b"power" in wos.lib().wos_last_error()


@pytest.mark.parametrize("case", ["forward", "backward_zero", "backward_tikhonov", "zero_distance"])
def test_noalloc_matches_oracle(case):
    """Against the FP64 oracle's asm_pad (optics/propagate.go:339-387) under
    the evanescent policies of optics/propagate.go:186-199."""
    ny, nx, dx, wl = 128, 256, 1e-6, 5e-7   # lambda / (2 dx) < 1: no evanescent bins ...
    if case != "forward":
        dx = 0.2e-6                          # ... here some, which backward steps zero or damp
    z = {"forward": 3e-4, "backward_zero": -2e-5, "backward_tikhonov": -2e-5, "zero_distance": 0.0}[case]
    ex = _field(ny, nx, dx, 5)
    kw = dict(wavelength=wl, backward_regularize=(case == "backward_tikhonov"))
    got = _run_noalloc(ex, dx, z, wos.Context(warnings_enabled=False, **kw))
    o = O.Field(ex.astype(np.complex128), dx)
    O.propagate(o, z, "asm_pad", O.Context(warnings_enabled=False, **kw))
    if case == "zero_distance":
        assert np.array_equal(got, ex.astype(np.complex128))
    assert rel_l2(got, o.ex) <= TOL_FP32, (case, rel_l2(got, o.ex))


def test_noalloc_in_place_and_smallest_grids():
    """in == out gives the out-of-place result; 4 x 4, 4 x 8 and 8 x 4 grids
    match the oracle."""
    dx, wl, z = 1e-6, 5e-7, 2e-5
    ctx = wos.Context(wavelength=wl, warnings_enabled=False)
    ex = _field(64, 128, dx, 7)
    a = _run_noalloc(ex, dx, z, ctx)
    b = _run_noalloc(ex, dx, z, ctx, inplace=True)
    assert np.array_equal(a, b)
    for ny, nx in ((4, 4), (4, 8), (8, 4)):
        ex = _field(ny, nx, dx, ny * 10 + nx)
        got = _run_noalloc(ex, dx, z, ctx)
        o = O.Field(ex.astype(np.complex128), dx)
        O.propagate(o, z, "asm_pad", O.Context(wavelength=wl, warnings_enabled=False))
        assert rel_l2(got, o.ex) <= TOL_FP32, ((ny, nx), rel_l2(got, o.ex))


def test_noalloc_calls_leave_device_memory_unchanged():
    """After one call per grid size (which loads the module and fills the
    twiddles), further calls on every size take no device memory: the free
    memory the driver reports is the same before and after them.  Measured
    twice if the first reading differs, in case another process on the GPU
    moved it."""
    import torch
    dx, wl, z = 1e-6, 5e-7, 2e-5
    sizes = ((4, 4), (64, 128), (1024, 1024), (512, 256))
    bufs = {s: (torch.zeros(s, dtype=torch.complex64, device="cuda"),
                torch.zeros(s, dtype=torch.complex64, device="cuda")) for s in sizes}
    for (ny, nx), (a, b) in bufs.items():
        assert _noalloc(a.data_ptr(), b.data_ptr(), ny, nx, dx, z, wl, 0) == 0, wos.lib().wos_last_error()
    torch.cuda.synchronize()

    def free_change():
        before = torch.cuda.mem_get_info()[0]
        for _ in range(4):
            for (ny, nx), (a, b) in bufs.items():
                assert _noalloc(a.data_ptr(), b.data_ptr(), ny, nx, dx, z, wl, 0) == 0
        torch.cuda.synchronize()
        return before - torch.cuda.mem_get_info()[0]

    d = free_change()
    if d != 0:
        d = free_change()
    assert d == 0, d
