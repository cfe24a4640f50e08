"""The zero-padded ASM entry point that allocates no device memory.

Some callers cannot call cudaMalloc: processes that reserve every byte of a
GPU up front behind their own allocator, or pipelines that cannot afford the
device-wide synchronisation of cudaFree.  wos_asm_pad_c64_noalloc serves them
from file-scope device arrays instead of a context workspace.  These checks
call it through the C ABI and compare it with the regular asm_pad entry point
(same tolerance as the other FP32 parity tests), on two calls in a row with
different inputs, and check that sizes beyond its static workspace are
rejected.  The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from gpu_util import TOL_FP32, rel_l2, wos

pytestmark = pytest.mark.gpu


def _noalloc(in_ptr, out_ptr, ny, nx, dx, z, wl, stream):
    cc = wos.Context(wavelength=wl, warnings_enabled=False).c()
    return wos.lib().wos_asm_pad_c64_noalloc(C.c_void_p(in_ptr), C.c_void_p(out_ptr), ny, nx, dx, z,
                                              C.byref(cc), C.c_void_p(stream))


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
