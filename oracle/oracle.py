"""TEST INFRASTRUCTURE ONLY: ctypes binding of the FP64 CPU oracle (wos_oracle.c).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module, and only as the checker.  The product library never calls it.

Fields are numpy complex128 arrays of shape (ny, nx), row-major, exactly the
memory layout of the reference's Field.Ex / Field.Ey (optics/field.go:14-22).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field as dfield
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libwos_oracle.so")

METHODS = {
    "asm": 1, "auto": 1, "": 1, "asm_pad": 2, "asm_shift": 3, "asm_shift_pad": 4,
    "fresnel_tf": 5, "fresnel_ir": 6, "fraunhofer": 7,
}


class _Warning(C.Structure):
    _fields_ = [("code", C.c_char * 32), ("count", C.c_int), ("value", C.c_double)]


class _Context(C.Structure):
    _fields_ = [
        ("wavelength", C.c_double), ("evanescent_zero", C.c_int),
        ("evanescent_limit", C.c_double), ("backward_regularize", C.c_int),
        ("tikhonov_alpha", C.c_double), ("has_warnings", C.c_int),
        ("n_warn", C.c_int), ("warn", _Warning * 16),
    ]


class _C128(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


def _c128(v) -> _C128:
    v = complex(v)
    return _C128(v.real, v.imag)


class _Field(C.Structure):
    _fields_ = [
        ("ny", C.c_int), ("nx", C.c_int), ("dx", C.c_double), ("polarized", C.c_int),
        ("ex", C.c_void_p), ("ey", C.c_void_p),
    ]


class IndexDesc(C.Structure):
    """Parametric n(x,y,z); identical layout to the product's wos_index_desc."""
    _fields_ = [
        ("re_bg", C.c_double), ("im_bg", C.c_double),
        ("core_dn", C.c_double), ("core_x0", C.c_double), ("core_y0", C.c_double),
        ("core_w", C.c_double), ("zmod_amp", C.c_double), ("zmod_period", C.c_double),
        ("zmod_phase", C.c_double), ("border_px", C.c_int), ("border_order", C.c_int),
        ("border_strength", C.c_double), ("n_layers", C.c_int),
        ("layer_z", C.c_double * 8), ("layer_re", C.c_double * 8), ("layer_im", C.c_double * 8),
    ]


def build() -> str:
    """Compile the oracle with its Makefile if the shared object is missing or stale."""
    src = os.path.join(HERE, "wos_oracle.c")
    if (not os.path.exists(LIB_PATH)) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        L.or_fft1d.argtypes = [vp, i, i]
        L.or_fft1d_pow2.argtypes = [vp, i, i]
        L.or_bluestein.argtypes = [vp, i, i]
        L.or_fft2d.argtypes = [vp, i, i, i]
        L.or_power.argtypes = [vp]; L.or_power.restype = d
        L.or_rms_radius.argtypes = [vp]; L.or_rms_radius.restype = d
        L.or_spectral_radius.argtypes = [vp, d]; L.or_spectral_radius.restype = d
        L.or_spectral_centroid.argtypes = [vp, vp, vp]
        L.or_propagate.argtypes = [vp, d, i, vp]; L.or_propagate.restype = i
        L.or_propagate_shift_at.argtypes = [vp, d, i, vp, d, d]; L.or_propagate_shift_at.restype = i
        L.or_propagate1d.argtypes = [vp, i, d, d, d, vp]
        L.or_propagate_vectorial.argtypes = [vp, vp, d, vp]
        L.or_propagate_uniaxial.argtypes = [vp, d, d, d, vp]
        L.or_propagate_uniaxial.restype = i
        L.or_propagate_anisotropic.argtypes = [vp, d, vp, vp]
        L.or_propagate_anisotropic.restype = i
        L.or_splitstep.argtypes = [vp, d, vp, i, vp]
        L.or_polychromatic.argtypes = [vp, d, vp, vp, i, i, vp, vp]; L.or_polychromatic.restype = i
        L.or_propagate3d.argtypes = [vp, vp, i, i, vp, vp]; L.or_propagate3d.restype = i
        L.or_schell_realizations.argtypes = [i, d, d, d, i, vp, vp]
        L.or_schell_realizations.restype = i
        L.or_average_intensity.argtypes = [vp, i, i, vp]
        L.or_hash_noise01.argtypes = [C.c_longlong] * 3; L.or_hash_noise01.restype = d
        L.or_apply_lens.argtypes = [vp, d, d, d, d, d]
        L.or_apply_aperture_circle.argtypes = [vp, d, d, d, d]
        L.or_apply_grating.argtypes = [vp, i, d, d, d, d, d, d]; L.or_apply_grating.restype = i
        L.or_apply_diffuser.argtypes = [vp, d, d, d, C.c_longlong, d, d]
        L.or_apply_phase_mask.argtypes = [vp, vp, d]
        L.or_apply_tilt.argtypes = [vp, d, d, d]
        L.or_apply_jones.argtypes = [vp, _C128, _C128, _C128, _C128]
        L.or_scale_amplitude.argtypes = [vp, _C128]
        L.or_apply_bandlimit.argtypes = [vp, d, d]
        L.or_shift_field.argtypes = [vp, d, d]
        L.or_index_eval.argtypes = [vp, i, i, d, i, i, d, d, d, vp, vp]
        L.or_asm_phase_loss_grad.argtypes = [i, i, d, d, vp, vp, vp, vp, vp]
        L.or_asm_phase_loss_grad.restype = d
        L.or_bpm_stack_loss_grad.argtypes = [i, i, d, i, vp, vp, vp, d, i, vp, vp, vp]
        L.or_bpm_stack_loss_grad.restype = d
        L.or_set_threads.argtypes = [i]
        L.or_get_threads.restype = i
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


@dataclass
class Context:
    """Mirror of optics.Context (field.go:237-254)."""
    wavelength: float
    evanescent: str = "decay"
    evanescent_limit: float = 0.0
    backward_regularize: bool = False
    tikhonov_alpha: float = 0.0
    warnings_enabled: bool = True
    warnings: dict = dfield(default_factory=dict)   # code -> (count, value)

    def _to_c(self) -> _Context:
        c = _Context()
        c.wavelength = self.wavelength
        c.evanescent_zero = 1 if self.evanescent == "zero" else 0
        c.evanescent_limit = self.evanescent_limit
        c.backward_regularize = 1 if self.backward_regularize else 0
        c.tikhonov_alpha = self.tikhonov_alpha
        c.has_warnings = 1 if self.warnings_enabled else 0
        c.n_warn = 0
        for code, (cnt, val) in self.warnings.items():
            w = c.warn[c.n_warn]
            w.code = code.encode()
            w.count = cnt
            w.value = val
            c.n_warn += 1
        return c

    def _from_c(self, c: _Context) -> None:
        self.warnings = {c.warn[k].code.decode(): (c.warn[k].count, c.warn[k].value)
                         for k in range(c.n_warn)}


class Field:
    """Mirror of optics.Field (field.go:14-22): ex/ey are (ny, nx) complex128."""

    def __init__(self, ex: np.ndarray, dx: float, ey: Optional[np.ndarray] = None):
        self.ex = np.ascontiguousarray(ex, dtype=np.complex128)
        self.ny, self.nx = self.ex.shape
        self.dx = float(dx)
        self.polarized = ey is not None
        self.ey = (np.ascontiguousarray(ey, dtype=np.complex128) if ey is not None
                   else np.zeros_like(self.ex))

    def clone(self) -> "Field":
        return Field(self.ex.copy(), self.dx, self.ey.copy() if self.polarized else None)

    def _c(self) -> _Field:
        f = _Field()
        f.ny, f.nx, f.dx, f.polarized = self.ny, self.nx, self.dx, int(self.polarized)
        f.ex, f.ey = _ptr(self.ex), _ptr(self.ey)
        return f

    def _sync(self, f: _Field) -> None:
        self.dx = f.dx
        self.polarized = bool(f.polarized)

    def x(self, i):
        return (np.asarray(i, dtype=np.float64) - self.nx / 2) * self.dx

    def y(self, j):
        return (np.asarray(j, dtype=np.float64) - self.ny / 2) * self.dx

    def intensity(self) -> np.ndarray:
        p = self.ex.real ** 2 + self.ex.imag ** 2
        if self.polarized:
            p = p + self.ey.real ** 2 + self.ey.imag ** 2
        return p

    def power(self) -> float:
        return lib().or_power(C.byref(self._c()))


def fft1d(a: np.ndarray, inverse: bool = False) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex128).copy()
    lib().or_fft1d(_ptr(a), a.size, int(inverse))
    return a


def fft2d(a: np.ndarray, inverse: bool = False) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex128).copy()
    lib().or_fft2d(_ptr(a), a.shape[0], a.shape[1], int(inverse))
    return a


def propagate(f: Field, z: float, method: str, ctx: Optional[Context]) -> None:
    """optics.Propagate (propagate.go:65-102), in place."""
    cf = f._c()
    if ctx is None:
        rc = lib().or_propagate(C.byref(cf), z, METHODS[method], None)
    else:
        cc = ctx._to_c()
        rc = lib().or_propagate(C.byref(cf), z, METHODS[method], C.byref(cc))
        ctx._from_c(cc)
    f._sync(cf)
    if rc != 0:
        raise ValueError(f"oracle propagate failed rc={rc}")


def propagate_shift_at(f: Field, z: float, method: str, ctx: Optional[Context], fxc: float, fyc: float) -> None:
    """propASMShift / propASMShiftPad (propagate.go:426-504) with the spectral
    centroid supplied instead of summed, in place."""
    cf = f._c()
    cc = ctx._to_c() if ctx is not None else None
    rc = lib().or_propagate_shift_at(C.byref(cf), z, METHODS[method], C.byref(cc) if cc is not None else None,
                                     fxc, fyc)
    if ctx is not None:
        ctx._from_c(cc)
    f._sync(cf)
    if rc != 0:
        raise ValueError(f"oracle propagate_shift_at failed rc={rc}")


def propagate1d(a: np.ndarray, dx: float, z: float, wl: float, ctx: Optional[Context]) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex128).copy()
    if ctx is None:
        lib().or_propagate1d(_ptr(a), a.size, dx, z, wl, None)
    else:
        cc = ctx._to_c()
        lib().or_propagate1d(_ptr(a), a.size, dx, z, wl, C.byref(cc))
        ctx._from_c(cc)
    return a


def propagate_vectorial(f: Field, z: float, ctx: Optional[Context]) -> np.ndarray:
    """PropagateVectorial (vectorial.go:14-80): Ex, Ey in place; returns Ez."""
    ez = np.zeros_like(f.ex)
    cf = f._c()
    if ctx is None:
        lib().or_propagate_vectorial(C.byref(cf), _ptr(ez), z, None)
    else:
        cc = ctx._to_c()
        lib().or_propagate_vectorial(C.byref(cf), _ptr(ez), z, C.byref(cc))
        ctx._from_c(cc)
    return ez


def propagate_uniaxial(f: Field, z: float, no: float, ne: float, ctx: Context) -> None:
    """PropagateUniaxial (birefringent.go:19-61), in place."""
    cc = ctx._to_c()
    if lib().or_propagate_uniaxial(C.byref(f._c()), z, no, ne, C.byref(cc)) != 0:
        raise ValueError("uniaxial: n_o and n_e must be > 0")


def propagate_anisotropic(f: Field, z: float, eps: np.ndarray, ctx: Context) -> None:
    """PropagateAnisotropic (berreman.go:13-36), Ex and Ey in place."""
    e = np.ascontiguousarray(eps, dtype=np.complex128).reshape(3, 3)
    cc = ctx._to_c()
    lib().or_propagate_anisotropic(C.byref(f._c()), z, _ptr(e), C.byref(cc))


def spectral_radius(f: Field, frac: float) -> float:
    return lib().or_spectral_radius(C.byref(f._c()), frac)


def spectral_centroid(f: Field):
    fx, fy = C.c_double(), C.c_double()
    lib().or_spectral_centroid(C.byref(f._c()), C.byref(fx), C.byref(fy))
    return fx.value, fy.value


def rms_radius(f: Field) -> float:
    return lib().or_rms_radius(C.byref(f._c()))


def splitstep(f: Field, z: float, desc: IndexDesc, steps: int, ctx: Optional[Context]) -> None:
    cf = f._c()
    if ctx is None:
        lib().or_splitstep(C.byref(cf), z, C.byref(desc), steps, None)
    else:
        cc = ctx._to_c()
        lib().or_splitstep(C.byref(cf), z, C.byref(desc), steps, C.byref(cc))
        ctx._from_c(cc)


def index_map(desc: IndexDesc, ny: int, nx: int, dx: float, z: float):
    """n(x,y,z) sampled on the grid through the oracle's descriptor evaluation."""
    re = np.empty((ny, nx)); im = np.empty((ny, nx))
    r, q = C.c_double(), C.c_double()
    for j in range(ny):
        y = (j - ny / 2) * dx
        for i in range(nx):
            x = (i - nx / 2) * dx
            lib().or_index_eval(C.byref(desc), ny, nx, dx, i, j, x, y, z, C.byref(r), C.byref(q))
            re[j, i] = r.value; im[j, i] = q.value
    return re, im


def polychromatic(f: Field, z: float, wls, weights, method: str, ctx: Optional[Context]) -> np.ndarray:
    wl = np.ascontiguousarray(wls, dtype=np.float64)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    out = np.zeros((f.ny, f.nx))
    cc = ctx._to_c() if ctx is not None else None
    rc = lib().or_polychromatic(C.byref(f._c()), z, _ptr(wl), _ptr(w), wl.size, METHODS[method],
                                C.byref(cc) if cc is not None else None, _ptr(out))
    if ctx is not None:
        ctx._from_c(cc)
    if rc != 0:
        raise ValueError(f"polychromatic rc={rc}")
    return out


def propagate3d(f: Field, zs, method: str, ctx: Optional[Context]) -> np.ndarray:
    zz = np.ascontiguousarray(zs, dtype=np.float64)
    ncomp = 2 if f.polarized else 1
    out = np.zeros((zz.size, ncomp, f.ny, f.nx), dtype=np.complex128)
    cc = ctx._to_c() if ctx is not None else None
    rc = lib().or_propagate3d(C.byref(f._c()), _ptr(zz), zz.size, METHODS[method],
                              C.byref(cc) if cc is not None else None, _ptr(out))
    if ctx is not None:
        ctx._from_c(cc)
    if rc != 0:
        raise ValueError(f"propagate3d rc={rc}")
    return out


def schell_realizations(n: int, dx: float, width: float, coherence: float, noise: np.ndarray):
    noise = np.ascontiguousarray(noise, dtype=np.complex128)
    m = noise.shape[0]
    out = np.zeros((m, n, n), dtype=np.complex128)
    rc = lib().or_schell_realizations(n, dx, width, coherence, m, _ptr(noise), _ptr(out))
    if rc != 0:
        raise ValueError(f"schell rc={rc}")
    return out


def average_intensity(fields: np.ndarray) -> np.ndarray:
    fields = np.ascontiguousarray(fields, dtype=np.complex128)
    m = fields.shape[0]
    out = np.zeros(fields.shape[1:])
    lib().or_average_intensity(_ptr(fields), m, int(np.prod(fields.shape[1:])), _ptr(out))
    return out


def hash_noise01(x: int, y: int, seed: int) -> float:
    return lib().or_hash_noise01(x, y, seed)


def apply_lens(f: Field, wl, focal, aperture=0.0, x0=0.0, y0=0.0):
    lib().or_apply_lens(C.byref(f._c()), wl, focal, aperture, x0, y0)


def apply_aperture_circle(f: Field, radius, x0=0.0, y0=0.0, edge_sigma=0.0):
    lib().or_apply_aperture_circle(C.byref(f._c()), radius, x0, y0, edge_sigma)


GRATING_KINDS = {"amplitude_sin": 0, "amplitude_binary": 1, "phase_sin": 2, "phase_binary": 3,
                 "blazed": 4}


def apply_grating(f: Field, kind, period, modulation=1.0, duty=0.5, blaze_depth=np.pi,
                  rotation=0.0, offset=0.0):
    rc = lib().or_apply_grating(C.byref(f._c()), GRATING_KINDS[kind], period, modulation, duty,
                                blaze_depth, rotation, offset)
    if rc != 0:
        raise ValueError("grating kind")


def apply_diffuser(f: Field, sigma=np.pi, corr=2e-5, amp=1.0, seed=1, x0=0.0, y0=0.0):
    lib().or_apply_diffuser(C.byref(f._c()), sigma, corr, amp, seed, x0, y0)


def apply_phase_mask(f: Field, phi: np.ndarray, amp=1.0):
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    lib().or_apply_phase_mask(C.byref(f._c()), _ptr(phi), amp)


def apply_jones(f: Field, a, b, c, d):
    cf = f._c()
    lib().or_apply_jones(C.byref(cf), _c128(a), _c128(b), _c128(c), _c128(d))
    f._sync(cf)


def scale_amplitude(f: Field, s):
    lib().or_scale_amplitude(C.byref(f._c()), _c128(s))


def apply_tilt(f: Field, tx, ty, wl):
    lib().or_apply_tilt(C.byref(f._c()), tx, ty, wl)


def apply_bandlimit(f: Field, fraction, sigma):
    lib().or_apply_bandlimit(C.byref(f._c()), fraction, sigma)


def shift_field(f: Field, du, dv):
    lib().or_shift_field(C.byref(f._c()), du, dv)


def asm_phase_loss_grad(a: np.ndarray, phi: np.ndarray, target: np.ndarray, dx: float, z: float,
                        ctx: Context, want_grad: bool = True):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    target = np.ascontiguousarray(target, dtype=np.float64)
    ny, nx = a.shape
    grad = np.zeros((ny, nx)) if want_grad else None
    cc = ctx._to_c()
    loss = lib().or_asm_phase_loss_grad(ny, nx, dx, z, C.byref(cc), _ptr(a), _ptr(phi),
                                        _ptr(target), _ptr(grad) if want_grad else None)
    return loss, grad


def bpm_stack_loss_grad(a: np.ndarray, phis: np.ndarray, target: np.ndarray, dx: float, zseg: float,
                        steps: int, desc: IndexDesc, ctx: Context, want_grad: bool = True):
    """Diffractive stack (masks phis[l] with a BPM segment of `steps` slices
    over zseg after each): loss sum (|u|^2 - T)^2 and dL/dphi per layer."""
    a = np.ascontiguousarray(a, dtype=np.complex128)
    phis = np.ascontiguousarray(phis, dtype=np.float64)
    target = np.ascontiguousarray(target, dtype=np.float64)
    nl, ny, nx = phis.shape
    grads = np.zeros((nl, ny, nx)) if want_grad else None
    cc = ctx._to_c()
    loss = lib().or_bpm_stack_loss_grad(ny, nx, dx, nl, _ptr(a), _ptr(phis), _ptr(target), zseg, steps,
                                        C.byref(desc), C.byref(cc), _ptr(grads) if want_grad else None)
    return loss, grads


def set_threads(p: int) -> None:
    lib().or_set_threads(int(p))


def get_threads() -> int:
    return lib().or_get_threads()


# ---------------------------------------------------------------------------
# Source construction used by the reference's tests: BuildSource "plane" and
# "gaussian" with tilt and power normalisation (optics/source.go:89-277).
# ---------------------------------------------------------------------------
def build_source(kind: str, n: int, width: float, wl: float, waist: float = 1e-3,
                 tilt_x: float = 0.0, tilt_y: float = 0.0, power: float = 1e-3,
                 x0: float = 0.0, y0: float = 0.0) -> Field:
    dx = width / n
    f = Field(np.zeros((n, n), dtype=np.complex128), dx)
    if kind == "plane":
        f.ex[:] = 1
    elif kind == "gaussian":
        xs = f.x(np.arange(n)) - x0
        ys = f.y(np.arange(n)) - y0
        r2 = xs[None, :] * xs[None, :] + ys[:, None] * ys[:, None]
        f.ex[:] = np.exp(-r2 / (waist * waist))
    else:
        raise ValueError(kind)
    if tilt_x != 0 or tilt_y != 0:
        apply_tilt(f, tilt_x, tilt_y, wl)
    cur = f.power()
    s = np.sqrt(power / cur)
    f.ex *= s
    return f


# ---- plane views (server/views.go:131-258) in the binary plane format
# (server/server.go:620-630: float32 little-endian, row-major, no header)
PHASE_MASK_CUT = 2e-3  # server/views.go:48


def plane_view(f: Field, view: str, ez: Optional[np.ndarray] = None, mask_cut: float = 0.0) -> np.ndarray:
    """One view of a field as the server's fmt=bin array (float32, little-endian)."""
    def n2(a):
        return a.real * a.real + a.imag * a.imag
    if view in ("total", "amplitude"):
        v = n2(f.ex)
        if f.polarized:
            v = v + n2(f.ey)
        if ez is not None:
            v = v + n2(ez)
        if view == "amplitude":
            v = np.sqrt(v)
    elif view in ("ex", "ey", "ez"):
        v = n2({"ex": f.ex, "ey": f.ey, "ez": ez}[view])
    else:
        src = {"phase_x": f.ex, "phase_y": f.ey, "phase_z": ez}[view]
        mc = mask_cut if mask_cut > 0 else PHASE_MASK_CUT
        p = n2(src)
        peak = p.max()
        v = np.arctan2(src.imag, src.real)
        v = np.where((peak <= 0) | (p < mc * peak), np.nan, v)
    return np.ascontiguousarray(v.astype("<f4"))
