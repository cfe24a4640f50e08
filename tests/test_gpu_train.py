"""Element train on the device (wos_train): the element loop of
trainer.runTrain (optics/simulator.go:397-500) with one upload and one
download per field.  Checked against the same sequence of oracle calls
(Propagate, the element Apply methods, ApplyBandlimit after every
propagation as runTrain does) and against one host call per op on the GPU.

Tolerances: FP64 1e-11 over a train of three propagations, FFT filters and
elements; FP32 5e-5 (several FP32 FFT round trips in sequence)."""
import numpy as np
import pytest

import oracle as O
from gpu_util import rel_l2, wos

pytestmark = pytest.mark.gpu

PRECS = [pytest.param(wos.FP64, id="fp64"), pytest.param(wos.FP32, id="fp32")]
WL = 632.8e-9
BL = (0.9, 0.05)


@pytest.fixture(scope="module", params=PRECS)
def gpu(request):
    g = wos.GPU(request.param)
    yield g
    g.close()


def _tol(prec):
    return 1e-11 if prec == wos.FP64 else 5e-5


def _ops(n, phi, sensor):
    return [
        ("lens", WL, 0.05, 100e-6, 3e-6, -2e-6),
        ("propagate", 4e-3, "asm"),
        ("aperture", 90e-6, 0.0, 0.0, 4e-6),
        ("propagate", 2e-3, "asm_pad"),
        ("grating", "phase_sin", 30e-6, 1.5, 0.5, 0.0, 0.2, 0.1),
        ("diffuser", 0.8, 8e-6, 0.95, 3, 1e-6, 0.0),
        ("phase_mask", phi, 0.9),
        ("jones", 0.8, 0.1j, 0.2, 0.7 - 0.1j),
        ("tilt", 0.002, -0.001, WL),
        ("intensity", sensor),
        ("shift", 3.5e-6, -2e-6),
        ("propagate", 3e-3, "fresnel_tf"),
        ("scale", 0.5 + 0.5j),
        ("bandlimit", 0.7, 0.1),
    ]


def _oracle_run(f, ops, ctx):
    sensor = None
    for op in ops:
        name, a = op[0], op[1:]
        if name == "propagate":
            O.propagate(f, a[0], a[1], ctx)
            O.apply_bandlimit(f, *BL)
        elif name == "lens":
            O.apply_lens(f, *a)
        elif name == "aperture":
            O.apply_aperture_circle(f, *a)
        elif name == "grating":
            O.apply_grating(f, *a)
        elif name == "diffuser":
            O.apply_diffuser(f, *a)
        elif name == "phase_mask":
            O.apply_phase_mask(f, a[0], a[1])
        elif name == "jones":
            O.apply_jones(f, *a)
        elif name == "tilt":
            O.apply_tilt(f, *a)
        elif name == "intensity":
            sensor = f.intensity().copy()
        elif name == "shift":
            O.shift_field(f, *a)
        elif name == "scale":
            O.scale_amplitude(f, a[0])
        elif name == "bandlimit":
            O.apply_bandlimit(f, *a)
    return sensor


@pytest.mark.parametrize("pol", [False, True])
def test_train_matches_oracle(gpu, pol):
    n, dx = 128, 2e-6
    rng = np.random.default_rng(11)
    ex = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    ey = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))) if pol else None
    phi = rng.uniform(0, 2 * np.pi, (n, n))
    of = O.Field(ex.copy(), dx, None if ey is None else ey.copy())
    oc = O.Context(wavelength=WL)
    want_sensor = _oracle_run(of, _ops(n, phi, None), oc)
    gf = wos.Field(ex.copy(), dx, None if ey is None else ey.copy())
    gc = wos.Context(wavelength=WL)
    sensor = np.zeros((n, n))
    gpu.train(gf, _ops(n, phi, sensor), gc, bandlimit=BL)
    t = _tol(gpu.precision)
    assert gf.polarized and of.polarized
    assert rel_l2(gf.ex, of.ex) <= t
    assert rel_l2(gf.ey, of.ey) <= t
    assert rel_l2(sensor, want_sensor) <= t
    assert set(gc.warnings) == set(oc.warnings)
    for k, (cnt, val) in oc.warnings.items():
        assert gc.warnings[k][0] == cnt, k


def test_train_equals_one_call_per_op(gpu):
    n, dx = 96, 2e-6
    rng = np.random.default_rng(2)
    ex = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    phi = rng.uniform(0, 2 * np.pi, (n, n))
    ops = [("lens", WL, 0.05, 0.0, 0.0, 0.0), ("propagate", 3e-3, "asm"), ("phase_mask", phi, 1.0),
           ("shift", 2e-6, 1e-6), ("propagate", 1e-3, "asm")]
    gf = wos.Field(ex.copy(), dx)
    gpu.train(gf, ops, wos.Context(wavelength=WL, warnings_enabled=False))
    hf = wos.Field(ex.copy(), dx)
    gpu.apply_lens(hf, WL, 0.05)
    gpu.propagate(hf, 3e-3, "asm", wos.Context(wavelength=WL, warnings_enabled=False))
    gpu.apply_phase_mask(hf, phi, 1.0)
    gpu.shift_field(hf, 2e-6, 1e-6)
    gpu.propagate(hf, 1e-3, "asm", wos.Context(wavelength=WL, warnings_enabled=False))
    assert rel_l2(gf.ex, hf.ex) <= 1e-14


def test_train_fraunhofer_pitch_carries_on(gpu):
    """The far-field step changes the pitch; the ops after it use the new one."""
    n, dx, z = 64, 4e-6, 0.5
    rng = np.random.default_rng(3)
    ex = np.exp(-((np.arange(n) - n / 2)[None, :] ** 2 + (np.arange(n) - n / 2)[:, None] ** 2) / 80.0) + 0j
    ex = ex * np.exp(1j * rng.uniform(0, 0.3, (n, n)))
    ops = [("propagate", z, "fraunhofer"), ("lens", WL, 0.2, 0.0, 0.0, 0.0), ("aperture", 2e-3, 0.0, 0.0, 0.0)]
    of = O.Field(ex.copy(), dx)
    O.propagate(of, z, "fraunhofer", O.Context(wavelength=WL))
    O.apply_lens(of, WL, 0.2)
    O.apply_aperture_circle(of, 2e-3)
    gf = wos.Field(ex.copy(), dx)
    gpu.train(gf, ops, wos.Context(wavelength=WL))
    assert gf.dx == pytest.approx(of.dx, rel=1e-15)
    assert rel_l2(gf.ex, of.ex) <= _tol(gpu.precision)


def test_train_argument_errors(gpu):
    ex = np.ones((32, 32), complex)
    with pytest.raises(wos.WosError):
        gpu.train(wos.Field(ex, 1e-6), [("propagate", 1e-3, "asm"), ("lens", WL, 0.0, 0.0, 0.0, 0.0)])
    with pytest.raises(KeyError):
        gpu.train(wos.Field(ex, 1e-6), [("teleport", 1.0)])
