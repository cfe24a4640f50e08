"""Three-sweep ASM through the tiled intermediate (FP32): the forward row
sweep stores columns in tiles of 4 contiguous per row block, the column sweep
reads each tile as one contiguous block, the inverse row sweep reads the tiles
back.  On by default in FP32 contexts; WOS_TILED=0 at context creation selects
the strided sweeps.  Compared with the oracle (FP32 tolerance 1e-5) and with
the strided sweeps on the same inputs (2e-6)."""
import os

import numpy as np
import pytest

import oracle as O
from gpu_util import TOL_FP32, rel_l2, wos

pytestmark = pytest.mark.gpu


def _ctx(tiled):
    old = os.environ.get("WOS_TILED")
    os.environ["WOS_TILED"] = "1" if tiled else "0"
    try:
        return wos.GPU(wos.FP32)
    finally:
        if old is None:
            del os.environ["WOS_TILED"]
        else:
            os.environ["WOS_TILED"] = old


@pytest.fixture(scope="module")
def pair():
    a, b = _ctx(True), _ctx(False)
    yield a, b
    a.close()
    b.close()


def _field(ny, nx, seed=1):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))


@pytest.mark.parametrize("shape", [(256, 256), (512, 128), (128, 1024)])
@pytest.mark.parametrize("pol", [False, True])
def test_tiled_propagate(pair, shape, pol):
    gt, g1 = pair
    ny, nx = shape
    dx, wl, z = 2e-6, 632.8e-9, 2e-4
    ex, ey = _field(ny, nx), _field(ny, nx, 2) if pol else None
    oc = O.Context(wavelength=wl)
    of = O.Field(ex.copy(), dx, None if ey is None else ey.copy())
    O.propagate(of, z, "asm", oc)
    res = []
    for g in (gt, g1):
        f = wos.Field(ex.copy(), dx, None if ey is None else ey.copy())
        gc = wos.Context(wavelength=wl)
        g.propagate(f, z, "asm", gc)
        assert rel_l2(f.ex, of.ex) <= TOL_FP32
        if pol:
            assert rel_l2(f.ey, of.ey) <= TOL_FP32
        assert set(gc.warnings) == set(oc.warnings)
        res.append(f)
    assert rel_l2(res[0].ex, res[1].ex) <= 2e-6


def test_tiled_evanescent_loss_sums(pair):
    gt, _ = pair
    ny, nx, dx, wl, z = 256, 512, 0.4e-6, 1e-6, 3e-6
    ex = _field(ny, nx, 3)
    oc = O.Context(wavelength=wl)
    of = O.Field(ex.copy(), dx)
    O.propagate(of, z, "asm", oc)
    f = wos.Field(ex.copy(), dx)
    gc = wos.Context(wavelength=wl)
    gt.propagate(f, z, "asm", gc)
    assert rel_l2(f.ex, of.ex) <= TOL_FP32
    for k, (cnt, val) in oc.warnings.items():
        assert gc.warnings[k][0] == cnt
        assert abs(gc.warnings[k][1] - val) <= 1e-4 * abs(val)


def test_tiled_device_batch_on_side_streams(pair):
    """Fields of a device batch on forked streams, each with its own tiled
    intermediate, equal the strided sweeps."""
    import torch
    gt, g1 = pair
    ny, nx, dx, wl, z = 2048, 2048, 2e-6, 632.8e-9, 5e-2
    rng = np.random.default_rng(5)
    fields = [torch.from_numpy(rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))).to(torch.complex64).cuda()
              for _ in range(5)]
    outs = {}
    for name, g in (("tiled", gt), ("strided", g1)):
        o = [torch.empty_like(t) for t in fields]
        torch.cuda.synchronize()
        g.propagate_batch_dev(ny, nx, dx, 1, [t.data_ptr() for t in fields], [t.data_ptr() for t in o], z, "asm",
                              wos.Context(wavelength=wl, warnings_enabled=False))
        g.synchronize()
        outs[name] = [t.cpu().numpy() for t in o]
    for a, b in zip(outs["tiled"], outs["strided"]):
        assert rel_l2(a, b) <= 2e-6
    # in place (in == out) through the tiled intermediate
    t0 = fields[0].clone()
    torch.cuda.synchronize()
    gt.propagate_dev(ny, nx, dx, 1, t0.data_ptr(), t0.data_ptr(), z, "asm",
                     wos.Context(wavelength=wl, warnings_enabled=False))
    gt.synchronize()
    assert rel_l2(t0.cpu().numpy(), outs["strided"][0]) <= 2e-6
