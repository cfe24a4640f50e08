"""Column sweep on two-CTA clusters (FP32, columns of 2048): each tile of 8
columns is split over a cluster, half a column per CTA, with the radix-2 steps
between the halves through distributed shared memory.  Enabled per context by
WOS_COLPAIR=1 at context creation; these tests compare it with the oracle and
with the single-CTA column sweep on the same inputs (FP32 tolerance 1e-5 against
the FP64 oracle; 2e-6 between the two FP32 sweeps)."""
import os

import numpy as np
import pytest

import oracle as O
from gpu_util import TOL_FP32, rel_l2, wos

pytestmark = pytest.mark.gpu


def _ctx(split):
    old = os.environ.get("WOS_COLPAIR")
    os.environ["WOS_COLPAIR"] = "1" if split else "0"
    try:
        return wos.GPU(wos.FP32)
    finally:
        if old is None:
            del os.environ["WOS_COLPAIR"]
        else:
            os.environ["WOS_COLPAIR"] = old


@pytest.fixture(scope="module")
def pair():
    a, b = _ctx(True), _ctx(False)
    yield a, b
    a.close()
    b.close()


def _field(ny, nx, seed=1):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))


@pytest.mark.parametrize("nx", [256, 64])
@pytest.mark.parametrize("z", [1e-3, -4e-4])
def test_split_tiles_propagate(pair, nx, z):
    gs, g1 = pair
    ny, dx, wl = 2048, 2e-6, 632.8e-9
    ex = _field(ny, nx)
    oc = O.Context(wavelength=wl)
    of = O.Field(ex.copy(), dx)
    O.propagate(of, z, "asm", oc)
    out = []
    for g in (gs, g1):
        f = wos.Field(ex.copy(), dx)
        gc = wos.Context(wavelength=wl)
        g.propagate(f, z, "asm", gc)
        out.append((f.ex, gc))
        assert rel_l2(f.ex, of.ex) <= TOL_FP32
        assert set(gc.warnings) == set(oc.warnings)
    assert rel_l2(out[0][0], out[1][0]) <= 2e-6


def test_split_tiles_evanescent_loss_sums(pair):
    """Evanescent bins present: the per-CTA loss sums of the split sweep give the
    reference's evanescent_filtered value."""
    gs, _ = pair
    ny, nx, dx, wl, z = 2048, 128, 0.4e-6, 1e-6, 3e-6
    ex = _field(ny, nx, 3)
    oc = O.Context(wavelength=wl)
    of = O.Field(ex.copy(), dx)
    O.propagate(of, z, "asm", oc)
    f = wos.Field(ex.copy(), dx)
    gc = wos.Context(wavelength=wl)
    gs.propagate(f, z, "asm", gc)
    assert rel_l2(f.ex, of.ex) <= TOL_FP32
    assert set(gc.warnings) == set(oc.warnings)
    for k, (cnt, val) in oc.warnings.items():
        assert gc.warnings[k][0] == cnt
        assert abs(gc.warnings[k][1] - val) <= 1e-4 * abs(val)


def test_split_tiles_device_batch(pair):
    """Device fields on the forked streams (the tables are built before the fork)."""
    import torch
    gs, g1 = pair
    ny, nx, dx, wl, z = 2048, 2048, 2e-6, 632.8e-9, 5e-2
    rng = np.random.default_rng(5)
    fields = [torch.from_numpy(rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))).to(torch.complex64).cuda()
              for _ in range(3)]
    outs = {}
    for name, g in (("split", gs), ("one", g1)):
        o = [torch.empty_like(t) for t in fields]
        torch.cuda.synchronize()
        g.propagate_batch_dev(ny, nx, dx, 1, [t.data_ptr() for t in fields], [t.data_ptr() for t in o], z, "asm",
                              wos.Context(wavelength=wl, warnings_enabled=False))
        g.synchronize()
        outs[name] = [t.cpu().numpy() for t in o]
    for a, b in zip(outs["split"], outs["one"]):
        assert rel_l2(a, b) <= 2e-6


def test_split_tiles_polychromatic_and_split_step(pair):
    """Batched units (shared row spectrum as the column source, per-unit
    wavelengths) and split-step slices on the split column sweep."""
    import torch
    gs, g1 = pair
    ny, nx, dx = 2048, 256, 1e-6
    ex = _field(ny, nx, 7)
    wls, wts = [500e-9, 600e-9, 700e-9], [1.0, 0.5, 0.25]
    ctx = wos.Context(wavelength=600e-9, warnings_enabled=False)
    i_s = gs.polychromatic(wos.Field(ex.copy(), dx), 1e-3, wls, wts, "asm", ctx)
    i_1 = g1.polychromatic(wos.Field(ex.copy(), dx), 1e-3, wls, wts, "asm", ctx)
    assert rel_l2(i_s, i_1) <= 2e-6
    d = wos.IndexDesc()
    d.re_bg, d.core_dn, d.core_w = 1.45, 0.01, 20e-6
    res = []
    for g in (gs, g1):
        buf = torch.from_numpy(ex).to(torch.complex64).cuda().contiguous()
        torch.cuda.synchronize()
        g.split_step_dev(ny, nx, dx, 1, buf.data_ptr(), 40e-6, d, 8, wos.Context(wavelength=1.55e-6,
                                                                              warnings_enabled=False))
        g.synchronize()
        res.append(buf.cpu().numpy())
    assert rel_l2(res[0], res[1]) <= 1e-5
