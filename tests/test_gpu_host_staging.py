"""Pageable host fields (plain numpy arrays, as Go slices are) go through
the library's page-locked staging with the conversion to the context
precision done on host threads; page-locked fields are copied directly.  The
two routes must give the same fields bit for bit, and the same warnings,
for single calls and batches, scalar and polarized, complex64 and
complex128 contexts."""
import numpy as np
import pytest
import torch

from gpu_util import wos

pytestmark = pytest.mark.gpu


def _fields(n, count, polarized, seed=9):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        ex = np.exp(1j * rng.uniform(0, 2 * np.pi, (n, n)))
        ey = 0.5 * np.exp(1j * rng.uniform(0, 2 * np.pi, (n, n))) if polarized else None
        out.append((ex, ey))
    return out


def _pinned(a):
    return torch.from_numpy(a.copy()).pin_memory().numpy()


@pytest.mark.parametrize("prec", [wos.FP64, wos.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("polarized", [False, True])
@pytest.mark.parametrize("method", ["asm", "asm_pad", "fraunhofer"])
def test_pageable_staging_equals_pinned_copies(prec, polarized, method):
    n, dx, wl = 256, 2e-6, 632.8e-9
    z = 0.5 if method == "fraunhofer" else 4e-3
    src = _fields(n, 5, polarized)
    with wos.GPU(prec) as g:
        res = {}
        for kind in ("pageable", "pinned"):
            conv = (lambda a: a.copy()) if kind == "pageable" else _pinned
            fs = []
            for ex, ey in src:
                f = wos.Field(ex, dx, ey)
                f.ex = conv(f.ex)
                f.ey = conv(f.ey)
                fs.append(f)
            ctx = wos.Context(wavelength=wl)
            g.propagate_batch(fs[:4], z, method, ctx)
            c1 = wos.Context(wavelength=wl)
            g.propagate(fs[4], z, method, c1)
            res[kind] = ([(f.ex.copy(), f.ey.copy(), f.dx) for f in fs], dict(ctx.warnings), dict(c1.warnings))
    a, b = res["pageable"], res["pinned"]
    for (ex1, ey1, dx1), (ex2, ey2, dx2) in zip(a[0], b[0]):
        assert np.array_equal(ex1, ex2)
        assert np.array_equal(ey1, ey2)
        assert dx1 == dx2
    assert a[1] == b[1] and a[2] == b[2]
