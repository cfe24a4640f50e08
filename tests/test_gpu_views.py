"""Plane views in the binary plane format (wos_plane_view / _dev and the
train's view op) against the oracle's restatement of server/views.go:
float32 bits identical for the intensity views (FP64 sums rounded once),
phase within one float32 ulp (CUDA's atan2 against the host's) with the same
NaN mask."""
import numpy as np
import pytest

import oracle as O
from gpu_util import wos

pytestmark = pytest.mark.gpu

PRECS = [pytest.param(wos.FP64, id="fp64"), pytest.param(wos.FP32, id="fp32")]


@pytest.fixture(scope="module", params=PRECS)
def gpu(request):
    g = wos.GPU(request.param)
    yield g
    g.close()


def _fields(ny=48, nx=80, seed=4):
    rng = np.random.default_rng(seed)
    c = lambda: rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))  # noqa: E731
    ex, ey, ez = c(), c(), c()
    ex[:, :10] *= 1e-3          # below the phase mask cut
    ey[5:9, :] = 0
    return ex, ey, ez


def _same(got, want, phase):
    gb, wb = got.view(np.uint32), want.view(np.uint32)
    nan_g, nan_w = np.isnan(got), np.isnan(want)
    assert np.array_equal(nan_g, nan_w)
    assert np.array_equal(gb[nan_g], wb[nan_w])          # 0x7fc00000
    ok = ~nan_g
    if phase:
        assert np.max(np.abs(gb[ok].astype(np.int64) - wb[ok].astype(np.int64))) <= 1
    else:
        assert np.array_equal(gb[ok], wb[ok])


VIEWS = ["total", "amplitude", "ex", "ey", "ez", "phase_x", "phase_y", "phase_z"]


@pytest.mark.parametrize("pol", [False, True])
@pytest.mark.parametrize("view", VIEWS)
def test_plane_view_matches_oracle(gpu, view, pol):
    ex, ey, ez = _fields()
    f = wos.Field(ex, 1e-6, ey if pol else None)
    of = O.Field(ex, 1e-6, ey if pol else None)
    if not pol:
        f.ey[:] = ey
        of.ey[:] = ey
    got = gpu.plane_view(f, view, ez)
    _same(got, O.plane_view(of, view, ez), view.startswith("phase"))


def test_plane_view_dark_component_is_all_nan(gpu):
    ex, ey, _ = _fields()
    f = wos.Field(ex, 1e-6, np.zeros_like(ey))
    got = gpu.plane_view(f, "phase_y")
    assert np.isnan(got).all()


def test_plane_view_device_and_train(gpu):
    import torch
    ex, ey, _ = _fields(64, 64, 7)
    f = wos.Field(ex.copy(), 1e-6, ey.copy())
    want = gpu.plane_view(f, "total")
    dt = torch.complex128 if gpu.precision == wos.FP64 else torch.complex64
    planes = torch.from_numpy(np.stack([ex, ey])).to(dt).cuda().contiguous()
    out = torch.empty((64, 64), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    gpu.plane_view_dev(64, 64, 2, planes.data_ptr(), None, "total", out.data_ptr())
    gpu.synchronize()
    got = out.cpu().numpy()
    if gpu.precision == wos.FP64:
        assert np.array_equal(got, want)
    else:
        assert np.max(np.abs(got - want) / np.abs(want).max()) <= 1e-6
    # the train's view op sees the field at its place in the train
    view = np.empty((64, 64), dtype=np.float32)
    g2 = wos.Field(ex.copy(), 1e-6, ey.copy())
    gpu.train(g2, [("view", "phase_x", view), ("scale", 2.0)])
    _same(view, O.plane_view(O.Field(ex, 1e-6, ey), "phase_x"), True)
    assert np.allclose(g2.ex, 2 * ex)


def test_plane_view_argument_errors(gpu):
    ex, _, _ = _fields(16, 16)
    with pytest.raises(wos.WosError):
        gpu.plane_view(wos.Field(ex, 1e-6), "ez")          # no Ez given
