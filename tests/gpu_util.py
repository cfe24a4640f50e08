"""Helpers shared by the GPU tests: the package under test and the oracle."""
import importlib
import json
import os

import numpy as np

wos = importlib.import_module("tetsuhiro-wos_b200")

# Tolerances (relative L2 against the FP64 oracle).
TOL_FP64 = 1e-12   # FP64 kernels
TOL_FP32 = 1e-5    # FP32 kernels (FP64 phase arguments)
# Non-power-of-two grids: the reference's Bluestein transform forms the chirp
# angle pi*k*k/n without reduction, so its own error grows with the length
# (1.6e-14 at n=100, 5.2e-13 at n=3000 against the exact DFT) and two correct
# FP64 propagations on such grids differ by up to ~2e-12.  FP64 parity there
# is held at 5e-12.
TOL_FP64_BLUESTEIN = 5e-12
# The carrier-shift methods (asm_shift, asm_shift_pad) have no constant floor:
# the last bits of the spectral centroid decide how the propagation phase
# k z sqrt(1 - rho^2) of the shifted bins rounds (a phase of ~1e4 rad, whose
# ulp is ~2e-12 rad): two ulps of the centroid move the 64^2 tilted field by
# 1.3e-12, and the reference's sequential sums move the 128^2 one by 4.5e-11.
# Their tests measure that floor per case instead (exact_centroid below).
# Gaussian-Schell synthesis takes sqrt(max(0, S)) of a spectrum whose tail is
# rounding noise (1414 of 4096 bins slightly negative at 64^2): the oracle and
# an independent FP64 restatement differ by 8.7e-9.
TOL_FP64_SCHELL = 1e-7
# Complex64 split-step BPM over many slices: the same transform pair is
# applied to a slowly changing field once per slice, and its single-precision
# rounding adds up coherently, 3.5e-8 per slice (measured on the 1024^2 cfg3
# medium against the FP64 path: 7.0e-6 / 1.39e-5 / 2.7e-5 / 5.4e-5 at 200 /
# 400 / 800 / 1600 slices over the same length; the same with no medium at
# all, so neither the screens nor H cause it).  Twiddles, rotation constants
# and H are applied as hi + lo pairs in these sweeps, which took the 400-slice
# error from 8.5e-5 to 1.39e-5; what remains is the FP32 arithmetic of the
# butterflies.  The bound of a run of S slices: 1e-5 up to 200 slices, else
# 5e-8 per slice.
def tol_fp32_splitstep(slices: int) -> float:
    return max(TOL_FP32, 5e-8 * slices)


def log_parity(case: str, precision, err: float, bound: float, **extra) -> None:
    """Append one measured error to the file named by WOS_PARITY_LOG (if set)."""
    path = os.environ.get("WOS_PARITY_LOG")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps(dict(case=case, precision="fp64" if precision == wos.FP64 else "fp32",
                                     rel_l2=err, bound=bound, **extra)) + "\n")


def rel_l2(a, b) -> float:
    den = np.sum(np.abs(b) ** 2)
    if den <= 0:
        return float(np.sqrt(np.sum(np.abs(a) ** 2)))
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) / den))


def tol(precision) -> float:
    return TOL_FP64 if precision == wos.FP64 else TOL_FP32


def is_pow2(n: int) -> bool:
    return n > 0 and (n & (n - 1)) == 0


def tol_case(precision, method: str, ny: int, nx: int) -> float:
    """Parity tolerance of one propagation case (see the floors above; lengths
    that are not powers of two take the Bluestein floor, which also covers the
    mixed-radix 2/3/5 transforms)."""
    if precision != wos.FP64:
        return TOL_FP32
    t = TOL_FP64
    if not (is_pow2(ny) and is_pow2(nx)) or (method in ("asm_pad", "asm_shift_pad", "fresnel_ir")
                                             and not (is_pow2(2 * ny) and is_pow2(2 * nx))):
        t = max(t, TOL_FP64_BLUESTEIN)
    return t


def exact_centroid(ex, ey, dx, with_scale=False):
    """spectralCentroid (optics/propagate.go:391-416) over the oracle's own
    spectrum, with every sum exactly rounded (math.fsum) instead of
    accumulated in sequence; frequencies as the reference's freq (index i
    <= n/2 positive).  with_scale: also the power-weighted mean |f| (of x and
    y, the larger), the scale of the sums' rounding (a centroid near zero
    comes from sums that cancel)."""
    import math

    import oracle as O

    ny, nx = ex.shape

    def freq(n):
        i = np.arange(n)
        return np.where(i <= n // 2, i, i - n) / (n * dx)

    fy, fx = freq(ny), freq(nx)
    w = np.zeros((ny, nx))
    for a in (ex,) if ey is None else (ex, ey):
        s = O.fft2d(a)
        w = w + (s.real * s.real + s.imag * s.imag)
    sw = math.fsum(w.ravel())
    if sw <= 0:
        return (0.0, 0.0, 0.0) if with_scale else (0.0, 0.0)
    cx = math.fsum((w * fx[None, :]).ravel()) / sw
    cy = math.fsum((w * fy[:, None]).ravel()) / sw
    if not with_scale:
        return cx, cy
    scale = max(float(np.sum(w * np.abs(fx)[None, :])), float(np.sum(w * np.abs(fy)[:, None]))) / sw
    return cx, cy, scale
