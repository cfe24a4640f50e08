"""ctypes binding of libwosgpu.so (include/wos_gpu.h) and a host mirror of the
reference `optics` interface for the propagation hot path.

The names follow the Go package: Context (optics/field.go:237-254), Field
(optics/field.go:14-22), propagate (optics/propagate.go:65-102),
propagate_split_step (optics/medium.go:22-45), propagate_polychromatic
(optics/polychromatic.go:18-44), propagate_3d (optics/volume.go:8-18),
generate_schell_realizations / propagate_partially_coherent
(optics/coherence.go:22-116).  Errors raise WosError; there is no CPU path:
if the shared library or a CUDA device is missing, calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field as dfield
from typing import Dict, Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libwosgpu.so")

METHODS = {"asm": 1, "auto": 1, "": 1, "asm_pad": 2, "asm_shift": 3, "asm_shift_pad": 4,
           "fresnel_tf": 5, "fresnel_ir": 6, "fraunhofer": 7}
FP64, FP32 = 0, 1
WARN_CODES = ["evanescent_filtered", "backward_regularized", "backward_evanescent",
              "asm_alias_wrap", "fresnel_tf_alias", "fresnel_ir_alias", "fraunhofer_nearfield"]
GRATING_KINDS = {"amplitude_sin": 0, "amplitude_binary": 1, "phase_sin": 2, "phase_binary": 3,
                 "blazed": 4}

# Every entry point of include/wos_gpu.h.
EXPORTS = [
    "wos_device_count", "wos_device_name", "wos_ctx_create", "wos_ctx_destroy",
    "wos_ctx_set_stream", "wos_ctx_get_stream", "wos_ctx_precision", "wos_ctx_set_col_width",
    "wos_ctx_synchronize", "wos_ctx_set_profiling", "wos_ctx_profile", "wos_ctx_profile_reset",
    "wos_ctx_launch_count", "wos_ctx_set_fast_path", "wos_autotune", "wos_ctx_set_tune", "wos_status_string", "wos_last_error", "wos_backend_info",
    "wos_fft2d", "wos_fft1d", "wos_fft2d_dev", "wos_propagate", "wos_propagate_dev",
    "wos_propagate_dev_c128", "wos_splitstep", "wos_splitstep_dev", "wos_splitstep_maps",
    "wos_polychromatic", "wos_volume", "wos_schell_modes", "wos_partially_coherent",
    "wos_apply_lens", "wos_apply_aperture_circle", "wos_apply_grating", "wos_apply_phase_mask",
    "wos_asm_forward_loss", "wos_asm_loss_grad", "wos_asm_loss_grad_dev", "wos_asm_adjoint",
    "wos_propagate_batch_dev", "wos_propagate_batch",
    "wos_asm_pad_c64_noalloc",
    "wos_apply_jones", "wos_scale_amplitude", "wos_apply_tilt", "wos_apply_bandlimit", "wos_shift_field",
    "wos_apply_diffuser", "wos_propagate1d",
    "wos_bpm_stack_loss_grad", "wos_bpm_stack_loss_grad_dev", "wos_splitstep_adjoint_dev",
    "wos_train", "wos_propagate_vectorial", "wos_plane_view", "wos_plane_view_dev",
    "wos_propagate_uniaxial", "wos_propagate_anisotropic",
    "wos_graph_capture_begin", "wos_graph_capture_fork", "wos_graph_capture_join", "wos_graph_capture_end",
    "wos_graph_launch", "wos_graph_destroy",
    "wos_splitstep_adjoint",
    "wos_polychromatic_dev", "wos_volume_dev", "wos_partially_coherent_dev",
    "wos_comm_unique_id", "wos_comm_init", "wos_comm_destroy", "wos_shard_range",
    "wos_polychromatic_sharded_dev", "wos_partially_coherent_sharded_dev", "wos_volume_sharded_dev",
]


class WosError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"wos status {status}: {msg}")
        self.status = status


class CContext(C.Structure):
    _fields_ = [("wavelength", C.c_double), ("evanescent_zero", C.c_int),
                ("evanescent_limit", C.c_double), ("backward_regularize", C.c_int),
                ("tikhonov_alpha", C.c_double), ("diagnostics", C.c_int)]


class CDiag(C.Structure):
    _fields_ = [("p_in", C.c_double), ("p_out", C.c_double), ("centroid_fx", C.c_double),
                ("centroid_fy", C.c_double), ("carrier_applied", C.c_int),
                ("wrap_checked", C.c_int), ("spectral_radius", C.c_double),
                ("rms_radius_in", C.c_double), ("dx_out", C.c_double),
                ("warn_count", C.c_int * 7), ("warn_value", C.c_double * 7)]


class C128(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


def _c128(v) -> C128:
    v = complex(v)
    return C128(v.real, v.imag)


class COp(C.Structure):
    _fields_ = [("kind", C.c_int), ("method", C.c_int), ("a", C.c_double * 8), ("m", C128 * 4),
                ("map", C.c_void_p), ("out", C.c_void_p)]


OP_KINDS = {"propagate": 1, "lens": 2, "aperture": 3, "grating": 4, "phase_mask": 5, "diffuser": 6,
            "jones": 7, "scale": 8, "tilt": 9, "shift": 10, "bandlimit": 11, "intensity": 12, "view": 13}
VIEWS = {"total": 0, "amplitude": 1, "ex": 2, "ey": 3, "ez": 4, "phase_x": 5, "phase_y": 6, "phase_z": 7}


class CField(C.Structure):
    _fields_ = [("ny", C.c_int), ("nx", C.c_int), ("dx", C.c_double), ("polarized", C.c_int),
                ("ex", C.c_void_p), ("ey", C.c_void_p)]


class IndexDesc(C.Structure):
    """wos_index_desc: parametric n(x,y,z) of a split-step medium."""
    _fields_ = [
        ("re_bg", C.c_double), ("im_bg", C.c_double),
        ("core_dn", C.c_double), ("core_x0", C.c_double), ("core_y0", C.c_double),
        ("core_w", C.c_double), ("zmod_amp", C.c_double), ("zmod_period", C.c_double),
        ("zmod_phase", C.c_double), ("border_px", C.c_int), ("border_order", C.c_int),
        ("border_strength", C.c_double), ("n_layers", C.c_int),
        ("layer_z", C.c_double * 8), ("layer_re", C.c_double * 8), ("layer_im", C.c_double * 8),
    ]


_lib = None


def lib():
    """Load libwosgpu.so; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise WosError(6, f"{LIB_PATH} is missing: run tetsuhiro-wos_b200/build.py")
        L = C.CDLL(LIB_PATH)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        P = C.POINTER
        sig = {
            "wos_device_count": ([], i), "wos_device_name": ([i, C.c_char_p, i], i),
            "wos_ctx_create": ([i, i, P(vp)], i), "wos_ctx_destroy": ([vp], i),
            "wos_ctx_set_stream": ([vp, vp], i), "wos_ctx_get_stream": ([vp], vp),
            "wos_ctx_precision": ([vp], i), "wos_ctx_set_col_width": ([vp, i], i),
            "wos_ctx_synchronize": ([vp], i), "wos_status_string": ([i], C.c_char_p),
            "wos_ctx_set_profiling": ([vp, i], i),
            "wos_ctx_profile": ([vp, i, P(d), P(C.c_longlong)], i),
            "wos_ctx_profile_reset": ([vp], i), "wos_ctx_launch_count": ([vp], C.c_longlong),
            "wos_ctx_set_fast_path": ([vp, i], i),
            "wos_autotune": ([vp, i, i, P(i), P(i), P(i)], i),
            "wos_ctx_set_tune": ([vp, i, i, i, i, i], i),
            "wos_last_error": ([], C.c_char_p), "wos_backend_info": ([], C.c_char_p),
            "wos_fft2d": ([vp, i, i, vp, i], i), "wos_fft1d": ([vp, i, vp, i], i),
            "wos_fft2d_dev": ([vp, i, i, i, vp, i], i),
            "wos_propagate": ([vp, vp, d, i, vp, vp], i),
            "wos_propagate_dev": ([vp, i, i, d, i, vp, vp, d, i, vp, vp], i),
            "wos_propagate_dev_c128": ([vp, i, i, d, i, vp, vp, d, i, vp, vp], i),
            "wos_splitstep": ([vp, vp, d, vp, i, vp, vp], i),
            "wos_splitstep_dev": ([vp, i, i, d, i, vp, d, vp, i, vp, vp], i),
            "wos_splitstep_maps": ([vp, vp, d, vp, vp, i, i, vp, vp], i),
            "wos_polychromatic": ([vp, vp, d, vp, vp, i, i, vp, vp, vp], i),
            "wos_volume": ([vp, vp, vp, i, i, vp, vp, vp], i),
            "wos_schell_modes": ([vp, i, d, d, d, i, vp, vp], i),
            "wos_partially_coherent": ([vp, i, d, d, d, i, vp, d, i, vp, vp, vp], i),
            "wos_apply_lens": ([vp, vp, d, d, d, d, d], i),
            "wos_apply_aperture_circle": ([vp, vp, d, d, d, d], i),
            "wos_apply_grating": ([vp, vp, i, d, d, d, d, d, d], i),
            "wos_apply_phase_mask": ([vp, vp, vp, d], i),
            "wos_asm_forward_loss": ([vp, i, i, d, d, vp, vp, vp, vp, vp], i),
            "wos_asm_loss_grad": ([vp, i, i, d, d, vp, vp, vp, vp, vp, vp], i),
            "wos_asm_loss_grad_dev": ([vp, i, i, d, d, vp, vp, vp, vp, vp, vp], i),
            "wos_propagate_batch_dev": ([vp, i, i, i, d, i, vp, vp, d, i, vp], i),
            "wos_propagate_batch": ([vp, i, vp, d, i, vp, vp], i),
            "wos_asm_adjoint": ([vp, vp, d, vp], i),
            "wos_asm_pad_c64_noalloc": ([vp, vp, i, i, d, d, vp, vp], i),
            "wos_apply_jones": ([vp, vp, C128, C128, C128, C128], i),
            "wos_scale_amplitude": ([vp, vp, C128], i),
            "wos_apply_tilt": ([vp, vp, d, d, d], i),
            "wos_apply_bandlimit": ([vp, vp, d, d], i),
            "wos_shift_field": ([vp, vp, d, d], i),
            "wos_apply_diffuser": ([vp, vp, d, d, d, C.c_longlong, d, d], i),
            "wos_propagate1d": ([vp, i, vp, d, d, d, vp, vp], i),
            "wos_bpm_stack_loss_grad": ([vp, i, i, d, i, vp, vp, vp, d, vp, i, vp, vp, vp], i),
            "wos_bpm_stack_loss_grad_dev": ([vp, i, i, d, i, vp, vp, vp, d, vp, i, vp, vp, vp], i),
            "wos_splitstep_adjoint_dev": ([vp, i, i, d, i, vp, d, vp, i, vp], i),
            "wos_train": ([vp, vp, vp, i, vp, d, d, vp], i),
            "wos_propagate_vectorial": ([vp, vp, vp, d, vp], i),
            "wos_plane_view": ([vp, vp, vp, i, d, vp], i),
            "wos_plane_view_dev": ([vp, i, i, i, vp, vp, i, d, vp], i),
            "wos_propagate_uniaxial": ([vp, vp, d, d, d, vp], i),
            "wos_propagate_anisotropic": ([vp, vp, d, vp, vp], i),
            "wos_graph_capture_begin": ([vp], i), "wos_graph_capture_end": ([vp, vp], i),
            "wos_graph_capture_fork": ([vp, vp], i), "wos_graph_capture_join": ([vp, vp], i),
            "wos_graph_launch": ([vp, vp], i), "wos_graph_destroy": ([vp], i),
            "wos_splitstep_adjoint": ([vp, vp, d, vp, i, vp], i),
            "wos_polychromatic_dev": ([vp, i, i, d, i, vp, d, vp, vp, i, vp, vp], i),
            "wos_volume_dev": ([vp, i, i, d, i, vp, vp, i, vp, vp], i),
            "wos_partially_coherent_dev": ([vp, i, d, d, d, i, vp, d, vp, vp], i),
            "wos_comm_unique_id": ([vp], i), "wos_comm_init": ([vp, i, i, vp], i), "wos_comm_destroy": ([vp], i),
            "wos_shard_range": ([i, i, i, P(i), P(i)], i),
            "wos_polychromatic_sharded_dev": ([vp, i, i, d, i, vp, d, vp, vp, i, vp, vp], i),
            "wos_partially_coherent_sharded_dev": ([vp, i, d, d, d, i, vp, d, vp, vp], i),
            "wos_volume_sharded_dev": ([vp, i, i, d, i, vp, vp, i, vp, vp], i),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise WosError(rc, lib().wos_last_error().decode(errors="replace"))


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


def _out_array(out, shape, dtype):
    """A caller-supplied output array (e.g. page-locked) after checking it, else a new one."""
    if out is None:
        return np.zeros(shape, dtype=dtype)
    if out.shape != tuple(shape) or out.dtype != dtype or not out.flags["C_CONTIGUOUS"]:
        raise WosError(1, f"output array must be C-contiguous {dtype.__name__} {tuple(shape)}")
    return out


def device_count() -> int:
    return lib().wos_device_count()


def comm_unique_id() -> bytes:
    """wos_comm_unique_id: the id rank 0 shares with the other ranks."""
    buf = (C.c_ubyte * 128)()
    _check(lib().wos_comm_unique_id(buf))
    return bytes(buf)


def shard_range(units: int, nranks: int, rank: int) -> Tuple[int, int]:
    """wos_shard_range: the contiguous units [begin, end) of one rank (host only)."""
    b, e = C.c_int(), C.c_int()
    _check(lib().wos_shard_range(units, nranks, rank, C.byref(b), C.byref(e)))
    return b.value, e.value


def backend_info() -> str:
    """GPUBackendInfo (optics/gpu.go:139-143)."""
    return lib().wos_backend_info().decode()


@dataclass
class Context:
    """optics.Context (field.go:237-254) with its Warnings list (code -> (count, value))."""
    wavelength: float
    evanescent: str = "decay"
    evanescent_limit: float = 0.0
    backward_regularize: bool = False
    tikhonov_alpha: float = 0.0
    warnings_enabled: bool = True
    warnings: Dict[str, Tuple[int, float]] = dfield(default_factory=dict)

    def c(self) -> CContext:
        cc = CContext()
        cc.wavelength = self.wavelength
        cc.evanescent_zero = 1 if self.evanescent == "zero" else 0
        cc.evanescent_limit = self.evanescent_limit
        cc.backward_regularize = 1 if self.backward_regularize else 0
        cc.tikhonov_alpha = self.tikhonov_alpha
        cc.diagnostics = 1 if self.warnings_enabled else 0
        return cc

    def absorb(self, d: CDiag) -> None:
        """Warnings.Add for every warning the call raised (field.go:322-338)."""
        if not self.warnings_enabled:
            return
        for b, code in enumerate(WARN_CODES):
            n = d.warn_count[b]
            if n <= 0:
                continue
            cnt, val = self.warnings.get(code, (0, 0.0))
            v = d.warn_value[b]
            self.warnings[code] = (cnt + n, v if v != 0 else val)


class Field:
    """optics.Field (field.go:14-22): ex/ey complex128 (ny, nx), row-major."""

    def __init__(self, ex: np.ndarray, dx: float, ey: Optional[np.ndarray] = None):
        self.ex = np.ascontiguousarray(ex, dtype=np.complex128)
        self.ny, self.nx = self.ex.shape
        self.dx = float(dx)
        self.polarized = ey is not None
        self.ey = (np.ascontiguousarray(ey, dtype=np.complex128) if ey is not None
                   else np.zeros_like(self.ex))

    def clone(self) -> "Field":
        return Field(self.ex.copy(), self.dx, self.ey.copy() if self.polarized else None)

    def c(self) -> CField:
        f = CField()
        f.ny, f.nx, f.dx, f.polarized = self.ny, self.nx, self.dx, int(self.polarized)
        f.ex, f.ey = _ptr(self.ex), _ptr(self.ey)
        return f

    def x(self, i):
        """X (field.go:59): centred column coordinate."""
        return (np.asarray(i, dtype=np.float64) - self.nx / 2) * self.dx

    def y(self, j):
        """Y (field.go:62): centred row coordinate."""
        return (np.asarray(j, dtype=np.float64) - self.ny / 2) * self.dx

    def intensity(self) -> np.ndarray:
        p = np.abs(self.ex) ** 2
        if self.polarized:
            p = p + np.abs(self.ey) ** 2
        return p

    def power(self) -> float:
        return float(self.intensity().sum() * self.dx * self.dx)


class Graph:
    """A captured sequence of device-resident calls (wos_graph), replayed with launch()."""

    def __init__(self, gpu: "GPU", h):
        self.gpu, self.h = gpu, h

    def launch(self) -> None:
        _check(lib().wos_graph_launch(self.gpu.h, self.h))

    def close(self) -> None:
        if self.h:
            lib().wos_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GPU:
    """One wos_ctx: a device, a precision (FP32 / FP64) and a CUDA stream."""

    def __init__(self, precision: int = FP32, device: int = 0):
        h = C.c_void_p()
        _check(lib().wos_ctx_create(device, precision, C.byref(h)))
        self.h = h
        self.precision = precision

    def close(self) -> None:
        if self.h:
            lib().wos_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return lib().wos_ctx_get_stream(self.h) or 0

    def set_stream(self, stream_ptr: int) -> None:
        _check(lib().wos_ctx_set_stream(self.h, C.c_void_p(stream_ptr)))

    def set_col_width(self, w: int) -> None:
        _check(lib().wos_ctx_set_col_width(self.h, w))

    def synchronize(self) -> None:
        _check(lib().wos_ctx_synchronize(self.h))

    PROFILE_KINDS = ["row_fwd", "row_inv", "row_inv_screen_fwd", "row_inv_accumulate",
                     "col_fused", "col_fraunhofer", "col_reduce", "col_fft"]

    def set_profiling(self, on: bool) -> None:
        _check(lib().wos_ctx_set_profiling(self.h, int(on)))

    def profile(self) -> dict:
        """{kind: (total_ms, launches)} of the per-launch CUDA-event profile."""
        out = {}
        for k, name in enumerate(self.PROFILE_KINDS):
            ms, n = C.c_double(), C.c_longlong()
            _check(lib().wos_ctx_profile(self.h, k, C.byref(ms), C.byref(n)))
            if n.value:
                out[name] = (ms.value, n.value)
        return out

    def profile_reset(self) -> None:
        _check(lib().wos_ctx_profile_reset(self.h))

    def launch_count(self) -> int:
        return int(lib().wos_ctx_launch_count(self.h))

    # ---- fft2D / fft1DAny users
    def fft2d(self, a: np.ndarray, inverse: bool = False) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.complex128).copy()
        _check(lib().wos_fft2d(self.h, a.shape[0], a.shape[1], _ptr(a), int(inverse)))
        return a

    def fft1d(self, a: np.ndarray, inverse: bool = False) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.complex128).copy()
        _check(lib().wos_fft1d(self.h, a.size, _ptr(a), int(inverse)))
        return a

    def fft2d_dev(self, ptr: int, ny: int, nx: int, batch: int = 1, inverse: bool = False) -> None:
        _check(lib().wos_fft2d_dev(self.h, ny, nx, batch, C.c_void_p(ptr), int(inverse)))

    # ---- Propagate
    def propagate(self, f: Field, z: float, method: str = "asm", ctx: Optional[Context] = None) -> CDiag:
        """optics.Propagate on a host field, in place (propagate.go:65-102)."""
        d = CDiag()
        cf = f.c()
        if method not in METHODS:
            raise WosError(7, f"unknown propagation method {method!r}")
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_propagate(self.h, C.byref(cf), z, METHODS[method],
                                   C.byref(cc) if cc is not None else None, C.byref(d)))
        if method == "fraunhofer" and z != 0:
            f.dx = d.dx_out
        if ctx is not None:
            ctx.absorb(d)
        return d

    def propagate_dev(self, ny: int, nx: int, dx: float, ncomp: int, in_ptr: int, out_ptr: int, z: float,
                      method: str, ctx: Optional[Context], diag: bool = False, c128: bool = False):
        d = CDiag() if diag else None
        cc = ctx.c() if ctx is not None else None
        fn = lib().wos_propagate_dev_c128 if c128 else lib().wos_propagate_dev
        _check(fn(self.h, ny, nx, dx, ncomp, C.c_void_p(in_ptr), C.c_void_p(out_ptr), z, METHODS[method],
                  C.byref(cc) if cc is not None else None, C.byref(d) if d is not None else None))
        if d is not None and ctx is not None:
            ctx.absorb(d)
        return d

    def propagate_batch(self, fields, z: float, method: str = "asm", ctx: Optional[Context] = None):
        """wos_propagate_batch: host fields in place, copies and sweeps of consecutive fields overlapped."""
        if method not in METHODS:
            raise WosError(7, f"unknown propagation method {method!r}")
        n = len(fields)
        cf = (CField * n)(*[f.c() for f in fields])
        ds = (CDiag * n)()
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_propagate_batch(self.h, n, cf, z, METHODS[method], C.byref(cc) if cc is not None else None,
                                         ds))
        for f, c_, d in zip(fields, cf, ds):
            if method == "fraunhofer":
                f.dx = c_.dx
            if ctx is not None:
                ctx.absorb(d)
        return list(ds)

    def propagate_batch_dev(self, ny: int, nx: int, dx: float, ncomp: int, in_ptrs, out_ptrs, z: float,
                            method: str, ctx: Optional[Context]) -> None:
        """wos_propagate_batch_dev: independent device fields, concurrently where the path allows."""
        n = len(in_ptrs)
        ia = (C.c_void_p * n)(*[C.c_void_p(p) for p in in_ptrs])
        oa = (C.c_void_p * n)(*[C.c_void_p(p) for p in out_ptrs])
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_propagate_batch_dev(self.h, n, ny, nx, dx, ncomp, ia, oa, z, METHODS[method],
                                             C.byref(cc) if cc is not None else None))

    # ---- PropagateSplitStep
    def split_step(self, f: Field, z: float, desc: IndexDesc, steps: int, ctx: Optional[Context]) -> CDiag:
        d = CDiag()
        cf = f.c()
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_splitstep(self.h, C.byref(cf), z, C.byref(desc), steps,
                                   C.byref(cc) if cc is not None else None, C.byref(d)))
        if ctx is not None:
            ctx.absorb(d)
        return d

    def split_step_maps(self, f: Field, z: float, n_re: np.ndarray, n_im: np.ndarray, steps: int,
                        ctx: Optional[Context]) -> CDiag:
        n_re = np.ascontiguousarray(n_re, dtype=np.float64)
        n_im = np.ascontiguousarray(n_im, dtype=np.float64)
        nmaps = 1 if n_re.ndim == 2 else n_re.shape[0]
        d = CDiag()
        cf = f.c()
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_splitstep_maps(self.h, C.byref(cf), z, _ptr(n_re), _ptr(n_im), nmaps, steps,
                                        C.byref(cc) if cc is not None else None, C.byref(d)))
        if ctx is not None:
            ctx.absorb(d)
        return d

    def split_step_dev(self, ny, nx, dx, ncomp, ptr, z, desc, steps, ctx, diag=False):
        d = CDiag() if diag else None
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_splitstep_dev(self.h, ny, nx, dx, ncomp, C.c_void_p(ptr), z, C.byref(desc), steps,
                                       C.byref(cc) if cc is not None else None,
                                       C.byref(d) if d is not None else None))
        return d

    # ---- batches (warnings of every unit accumulate into ctx, like the shared ctx.Warnings)
    def polychromatic(self, f: Field, z: float, wavelengths, weights, method: str = "asm",
                      ctx: Optional[Context] = None, out: Optional[np.ndarray] = None) -> np.ndarray:
        """PropagatePolychromatic (polychromatic.go:18-44); `out` (float64 (ny, nx)) may be supplied."""
        wl = np.ascontiguousarray(wavelengths, dtype=np.float64)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        out = _out_array(out, (f.ny, f.nx), np.float64)
        d = CDiag()
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_polychromatic(self.h, C.byref(f.c()), z, _ptr(wl), _ptr(w), wl.size, METHODS[method],
                                       C.byref(cc) if cc is not None else None, _ptr(out), C.byref(d)))
        if ctx is not None:
            ctx.absorb(d)
        return out

    def volume(self, f: Field, zs, method: str = "asm", ctx: Optional[Context] = None,
               out: Optional[np.ndarray] = None) -> np.ndarray:
        """Propagate3D (volume.go:8-18): (nz, ncomp, ny, nx) complex128; `out` may be supplied."""
        zz = np.ascontiguousarray(zs, dtype=np.float64)
        ncomp = 2 if f.polarized else 1
        out = _out_array(out, (zz.size, ncomp, f.ny, f.nx), np.complex128)
        d = CDiag()
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_volume(self.h, C.byref(f.c()), _ptr(zz), zz.size, METHODS[method],
                                C.byref(cc) if cc is not None else None, _ptr(out), C.byref(d)))
        if ctx is not None:
            ctx.absorb(d)
        return out

    def schell_modes(self, n: int, dx: float, width: float, coherence: float, noise: np.ndarray) -> np.ndarray:
        """GenerateSchellRealizations (coherence.go:22-80) with caller noise."""
        noise = np.ascontiguousarray(noise, dtype=np.complex128)
        m = noise.shape[0]
        out = np.zeros((m, n, n), dtype=np.complex128)
        _check(lib().wos_schell_modes(self.h, n, dx, width, coherence, m, _ptr(noise), _ptr(out)))
        return out

    def partially_coherent(self, n: int, dx: float, width: float, coherence: float, noise: np.ndarray,
                           z: float, method: str = "asm", ctx: Optional[Context] = None,
                           out: Optional[np.ndarray] = None) -> np.ndarray:
        """PropagatePartiallyCoherent (coherence.go:105-116); `out` (float64 (n, n)) may be supplied."""
        noise = np.ascontiguousarray(noise, dtype=np.complex128)
        m = noise.shape[0]
        out = _out_array(out, (n, n), np.float64)
        d = CDiag()
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_partially_coherent(self.h, n, dx, width, coherence, m, _ptr(noise), z, METHODS[method],
                                            C.byref(cc) if cc is not None else None, _ptr(out), C.byref(d)))
        if ctx is not None:
            ctx.absorb(d)
        return out

    # ---- device-resident batches (device pointers; no diagnostics)
    def polychromatic_dev(self, ny: int, nx: int, dx: float, ncomp: int, field_ptr: int, z: float, wavelengths,
                          weights, ctx: Optional[Context], out_ptr: int) -> None:
        """wos_polychromatic_dev: out (device FP64 [ny][nx]) = sum_k w_k |U_k|^2."""
        wl = np.ascontiguousarray(wavelengths, dtype=np.float64)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_polychromatic_dev(self.h, ny, nx, dx, ncomp, C.c_void_p(field_ptr), z, _ptr(wl), _ptr(w),
                                           wl.size, C.byref(cc) if cc is not None else None, C.c_void_p(out_ptr)))

    def volume_dev(self, ny: int, nx: int, dx: float, ncomp: int, field_ptr: int, zs, ctx: Optional[Context],
                   out_ptr: int) -> None:
        """wos_volume_dev: out (device [nz][ncomp][ny][nx], context type)."""
        zz = np.ascontiguousarray(zs, dtype=np.float64)
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_volume_dev(self.h, ny, nx, dx, ncomp, C.c_void_p(field_ptr), _ptr(zz), zz.size,
                                    C.byref(cc) if cc is not None else None, C.c_void_p(out_ptr)))

    def partially_coherent_dev(self, n: int, dx: float, width: float, coherence: float, m: int, noise_ptr: int,
                               z: float, ctx: Optional[Context], out_ptr: int) -> None:
        """wos_partially_coherent_dev: noise device complex128 [m][n][n]; out device FP64 [n][n]."""
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_partially_coherent_dev(self.h, n, dx, width, coherence, m, C.c_void_p(noise_ptr), z,
                                                C.byref(cc) if cc is not None else None, C.c_void_p(out_ptr)))

    # ---- batches sharded over GPUs (collectives over the context's communicator)
    def comm_init(self, nranks: int, rank: int, uid: bytes) -> None:
        """wos_comm_init with the id from comm_unique_id() on rank 0."""
        buf = (C.c_ubyte * 128).from_buffer_copy(uid)
        _check(lib().wos_comm_init(self.h, nranks, rank, buf))

    def comm_destroy(self) -> None:
        _check(lib().wos_comm_destroy(self.h))

    def polychromatic_sharded_dev(self, ny, nx, dx, ncomp, field_ptr, z, wavelengths, weights, ctx, out_ptr):
        wl = np.ascontiguousarray(wavelengths, dtype=np.float64)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_polychromatic_sharded_dev(self.h, ny, nx, dx, ncomp, C.c_void_p(field_ptr), z, _ptr(wl),
                                                   _ptr(w), wl.size, C.byref(cc) if cc is not None else None,
                                                   C.c_void_p(out_ptr)))

    def partially_coherent_sharded_dev(self, n, dx, width, coherence, m, noise_ptr, z, ctx, out_ptr):
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_partially_coherent_sharded_dev(self.h, n, dx, width, coherence, m, C.c_void_p(noise_ptr), z,
                                                        C.byref(cc) if cc is not None else None, C.c_void_p(out_ptr)))

    def volume_sharded_dev(self, ny, nx, dx, ncomp, field_ptr, zs, ctx, out_ptr):
        zz = np.ascontiguousarray(zs, dtype=np.float64)
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_volume_sharded_dev(self.h, ny, nx, dx, ncomp, C.c_void_p(field_ptr), _ptr(zz), zz.size,
                                            C.byref(cc) if cc is not None else None, C.c_void_p(out_ptr)))

    # ---- launch configuration
    def set_fast_path(self, on) -> None:
        """0/False: general sweeps; 1/True: specialised sweeps with the column
        sweep pipelined where the layout allows (default); 2: specialised
        one-shot sweeps only; 3: row and column sweeps pipelined."""
        _check(lib().wos_ctx_set_fast_path(self.h, int(on)))

    def autotune(self, ny: int, nx: int) -> tuple:
        r, c, w = C.c_int(), C.c_int(), C.c_int()
        _check(lib().wos_autotune(self.h, ny, nx, C.byref(r), C.byref(c), C.byref(w)))
        return r.value, c.value, w.value

    def set_tune(self, ny: int, nx: int, row_e: int, col_e: int, col_w: int) -> None:
        _check(lib().wos_ctx_set_tune(self.h, ny, nx, row_e, col_e, col_w))

    # ---- thin elements
    def apply_lens(self, f: Field, wl, focal, aperture=0.0, x0=0.0, y0=0.0):
        _check(lib().wos_apply_lens(self.h, C.byref(f.c()), wl, focal, aperture, x0, y0))

    def apply_aperture_circle(self, f: Field, radius, x0=0.0, y0=0.0, edge_sigma=0.0):
        _check(lib().wos_apply_aperture_circle(self.h, C.byref(f.c()), radius, x0, y0, edge_sigma))

    def apply_grating(self, f: Field, kind, period, modulation=1.0, duty=0.5, blaze_depth=np.pi,
                      rotation=0.0, offset=0.0):
        _check(lib().wos_apply_grating(self.h, C.byref(f.c()), GRATING_KINDS[kind], period, modulation, duty,
                                       blaze_depth, rotation, offset))

    def apply_phase_mask(self, f: Field, phi: np.ndarray, amp=1.0):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        _check(lib().wos_apply_phase_mask(self.h, C.byref(f.c()), _ptr(phi), amp))

    # ---- field operations (field.go:109-168,199-228,264-294; elements.go:722-783)
    def apply_jones(self, f: Field, a, b, c, d):
        cf = f.c()
        _check(lib().wos_apply_jones(self.h, C.byref(cf), _c128(a), _c128(b), _c128(c), _c128(d)))
        f.polarized = bool(cf.polarized)

    def scale_amplitude(self, f: Field, s):
        _check(lib().wos_scale_amplitude(self.h, C.byref(f.c()), _c128(s)))

    def apply_tilt(self, f: Field, tx, ty, wl):
        _check(lib().wos_apply_tilt(self.h, C.byref(f.c()), tx, ty, wl))

    def apply_bandlimit(self, f: Field, fraction, sigma):
        _check(lib().wos_apply_bandlimit(self.h, C.byref(f.c()), fraction, sigma))

    def shift_field(self, f: Field, du, dv):
        _check(lib().wos_shift_field(self.h, C.byref(f.c()), du, dv))

    def apply_diffuser(self, f: Field, sigma=np.pi, corr=2e-5, amp=1.0, seed=1, x0=0.0, y0=0.0):
        _check(lib().wos_apply_diffuser(self.h, C.byref(f.c()), sigma, corr, amp, int(seed), x0, y0))

    def propagate1d(self, a: np.ndarray, dx: float, z: float, wl: float, ctx: Optional[Context] = None,
                    diag: bool = False):
        """Propagate1D (propagate.go:718-738) on a copy of `a`; returns the
        propagated line (and the CDiag when diag is set)."""
        a = np.ascontiguousarray(a, dtype=np.complex128).copy()
        d = CDiag()
        cc = (ctx if ctx is not None else Context(wavelength=wl)).c()
        _check(lib().wos_propagate1d(self.h, a.size, _ptr(a), dx, z, wl, C.byref(cc), C.byref(d)))
        if ctx is not None:
            ctx.absorb(d)
        return (a, d) if diag else a

    def propagate_vectorial(self, f: Field, z: float, ctx: Optional[Context] = None) -> np.ndarray:
        """PropagateVectorial (vectorial.go:14-80): Ex, Ey in place; returns Ez."""
        ez = np.zeros_like(f.ex)
        cc = ctx.c() if ctx is not None else None
        _check(lib().wos_propagate_vectorial(self.h, C.byref(f.c()), _ptr(ez), z,
                                             C.byref(cc) if cc is not None else None))
        return ez

    # ---- CUDA graphs of device-resident calls
    def graph_capture_begin(self) -> None:
        _check(lib().wos_graph_capture_begin(self.h))

    def graph_capture_fork(self, other: "GPU") -> None:
        """wos_graph_capture_fork: other's calls become a concurrent branch of this capture."""
        _check(lib().wos_graph_capture_fork(self.h, other.h))

    def graph_capture_join(self, other: "GPU") -> None:
        """wos_graph_capture_join: close the branch forked to other."""
        _check(lib().wos_graph_capture_join(self.h, other.h))

    def graph_capture_end(self) -> "Graph":
        h = C.c_void_p()
        _check(lib().wos_graph_capture_end(self.h, C.byref(h)))
        return Graph(self, h)

    def propagate_uniaxial(self, f: Field, z: float, no: float, ne: float, ctx: Context) -> None:
        """PropagateUniaxial (birefringent.go:19-61), in place."""
        cc = ctx.c()
        _check(lib().wos_propagate_uniaxial(self.h, C.byref(f.c()), z, no, ne, C.byref(cc)))

    def propagate_anisotropic(self, f: Field, z: float, eps: np.ndarray, ctx: Context) -> None:
        """PropagateAnisotropic (berreman.go:13-36), Ex and Ey in place."""
        e = np.ascontiguousarray(eps, dtype=np.complex128).reshape(3, 3)
        cc = ctx.c()
        _check(lib().wos_propagate_anisotropic(self.h, C.byref(f.c()), z, _ptr(e), C.byref(cc)))

    def plane_view(self, f: Field, view: str, ez: Optional[np.ndarray] = None, mask_cut: float = 0.0) -> np.ndarray:
        """Binary plane format view (server fmt=bin): float32 (ny, nx)."""
        out = np.empty((f.ny, f.nx), dtype=np.float32)
        ezp = None
        if ez is not None:
            ez = np.ascontiguousarray(ez, dtype=np.complex128)
            ezp = _ptr(ez)
        _check(lib().wos_plane_view(self.h, C.byref(f.c()), ezp, VIEWS[view], mask_cut, _ptr(out)))
        return out

    def plane_view_dev(self, ny: int, nx: int, ncomp: int, planes_ptr: int, ez_ptr: Optional[int], view: str,
                       out_ptr: int, mask_cut: float = 0.0) -> None:
        _check(lib().wos_plane_view_dev(self.h, ny, nx, ncomp, C.c_void_p(planes_ptr),
                                        C.c_void_p(ez_ptr) if ez_ptr else None, VIEWS[view], mask_cut,
                                        C.c_void_p(out_ptr)))

    # ---- element train on the device (trainer.runTrain, simulator.go:397-500)
    def train(self, f: Field, ops, ctx: Optional[Context] = None, bandlimit=None, diag: bool = False):
        """Run `ops` on the field with one upload and one download.  Each op is
        a tuple: ("propagate", z, method), ("lens", wl, focal, aperture, x0, y0),
        ("aperture", radius, x0, y0, edge_sigma), ("grating", kind, period,
        modulation, duty, blaze_depth, rotation, offset), ("phase_mask", phi, amp),
        ("diffuser", sigma, corr, amp, seed, x0, y0), ("jones", a, b, c, d),
        ("scale", s), ("tilt", tx, ty, wl), ("shift", du, dv), ("bandlimit",
        fraction, sigma), ("intensity", out) with out a float64 (ny, nx) array.
        bandlimit = (fraction, sigma) is applied after every propagation."""
        arr = (COp * max(1, len(ops)))()
        keep = []
        for k, op in enumerate(ops):
            name, args = op[0], op[1:]
            o = arr[k]
            o.kind = OP_KINDS[name]
            if name == "propagate":
                o.a[0] = args[0]
                o.method = METHODS[args[1] if len(args) > 1 else "asm"]
            elif name == "grating":
                o.method = GRATING_KINDS[args[0]]
                for j, v in enumerate(args[1:]):
                    o.a[j] = v
            elif name == "phase_mask":
                phi = np.ascontiguousarray(args[0], dtype=np.float64)
                keep.append(phi)
                o.map = phi.ctypes.data
                o.a[0] = args[1] if len(args) > 1 else 1.0
            elif name == "intensity":
                out = args[0]
                assert out.dtype == np.float64 and out.flags["C_CONTIGUOUS"] and out.shape == (f.ny, f.nx)
                o.out = out.ctypes.data
            elif name == "view":
                o.method = VIEWS[args[0]]
                out = args[1]
                assert out.dtype == np.float32 and out.flags["C_CONTIGUOUS"] and out.shape == (f.ny, f.nx)
                o.out = out.ctypes.data
                o.a[0] = args[2] if len(args) > 2 else 0.0
            elif name in ("jones", "scale"):
                for j, v in enumerate(args):
                    o.m[j] = _c128(v)
            else:
                for j, v in enumerate(args):
                    o.a[j] = v
        d = CDiag()
        cf = f.c()
        cc = ctx.c() if ctx is not None else None
        fr, sg = bandlimit if bandlimit is not None else (0.0, 0.0)
        _check(lib().wos_train(self.h, C.byref(cf), arr, len(ops), C.byref(cc) if cc is not None else None, fr, sg,
                               C.byref(d) if (diag or ctx is not None) else None))
        f.polarized = bool(cf.polarized)
        f.dx = cf.dx
        if ctx is not None:
            ctx.absorb(d)
        return d

    # ---- diffractive stack (masks with BPM segments between them)
    def bpm_stack_loss_grad(self, a: np.ndarray, phis: np.ndarray, target: np.ndarray, dx: float, zseg: float,
                            steps: int, desc: "IndexDesc", ctx: Context, want_grad: bool = True):
        """Loss sum (|u|^2 - T)^2 of the stack and dL/dphi per layer (host arrays)."""
        a = np.ascontiguousarray(a, dtype=np.complex128)
        phis = np.ascontiguousarray(phis, dtype=np.float64)
        target = np.ascontiguousarray(target, dtype=np.float64)
        nl, ny, nx = phis.shape
        loss = C.c_double()
        grads = np.zeros((nl, ny, nx)) if want_grad else None
        cc = ctx.c()
        _check(lib().wos_bpm_stack_loss_grad(self.h, ny, nx, dx, nl, _ptr(a), _ptr(phis), _ptr(target), zseg,
                                             C.byref(desc), steps, C.byref(cc), C.byref(loss),
                                             _ptr(grads) if want_grad else None))
        return loss.value, grads

    def bpm_stack_loss_grad_dev(self, a_ptr: int, phis_ptr: int, target_ptr: int, grads_ptr: Optional[int],
                                nl: int, ny: int, nx: int, dx: float, zseg: float, steps: int, desc: "IndexDesc",
                                ctx: Context) -> float:
        """Device-resident stack loss / gradient: pointers to device arrays
        (a of the context's complex type; phis, target, grads FP64)."""
        loss = C.c_double()
        cc = ctx.c()
        _check(lib().wos_bpm_stack_loss_grad_dev(self.h, ny, nx, dx, nl, C.c_void_p(a_ptr), C.c_void_p(phis_ptr),
                                                 C.c_void_p(target_ptr), zseg, C.byref(desc), steps, C.byref(cc),
                                                 C.byref(loss), C.c_void_p(grads_ptr) if grads_ptr else None))
        return loss.value

    def split_step_adjoint(self, f: Field, z: float, desc: "IndexDesc", steps: int, ctx: Context) -> None:
        """Backward BPM: the adjoint of split_step on a host field, in place."""
        cc = ctx.c()
        _check(lib().wos_splitstep_adjoint(self.h, C.byref(f.c()), z, C.byref(desc), steps, C.byref(cc)))

    def split_step_adjoint_dev(self, ny, nx, dx, ncomp, ptr, z, desc, steps, ctx) -> None:
        """Adjoint of split_step_dev on a device field, in place."""
        cc = ctx.c()
        _check(lib().wos_splitstep_adjoint_dev(self.h, ny, nx, dx, ncomp, C.c_void_p(ptr), z, C.byref(desc), steps,
                                               C.byref(cc)))

    # ---- inverse design
    def asm_loss_grad(self, a: np.ndarray, phi: np.ndarray, target: np.ndarray, dx: float, z: float,
                      ctx: Context, want_grad: bool = True):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        target = np.ascontiguousarray(target, dtype=np.float64)
        ny, nx = a.shape
        loss = C.c_double()
        cc = ctx.c()
        if want_grad:
            grad = np.zeros((ny, nx))
            _check(lib().wos_asm_loss_grad(self.h, ny, nx, dx, z, C.byref(cc), _ptr(a), _ptr(phi), _ptr(target),
                                           C.byref(loss), _ptr(grad)))
            return loss.value, grad
        _check(lib().wos_asm_forward_loss(self.h, ny, nx, dx, z, C.byref(cc), _ptr(a), _ptr(phi), _ptr(target),
                                          C.byref(loss)))
        return loss.value, None

    def asm_loss_grad_dev(self, ny: int, nx: int, dx: float, z: float, ctx: Context, a_ptr: int, phi_ptr: int,
                          target_ptr: int, grad_ptr: int = 0) -> float:
        """wos_asm_loss_grad_dev: device arrays in, loss out (grad written on the device)."""
        loss = C.c_double()
        cc = ctx.c()
        _check(lib().wos_asm_loss_grad_dev(self.h, ny, nx, dx, z, C.byref(cc), C.c_void_p(a_ptr),
                                           C.c_void_p(phi_ptr), C.c_void_p(target_ptr), C.byref(loss),
                                           C.c_void_p(grad_ptr) if grad_ptr else None))
        return loss.value

    def asm_adjoint(self, f: Field, z: float, ctx: Context) -> None:
        cc = ctx.c()
        _check(lib().wos_asm_adjoint(self.h, C.byref(f.c()), z, C.byref(cc)))
