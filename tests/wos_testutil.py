"""Test fixtures restated from the reference's Go test helpers.

Each helper names the reference test file:line it follows.  Inputs are seeded
and deterministic; nothing here calls the product library.
"""
from __future__ import annotations

import math

import numpy as np

MASK64 = (1 << 64) - 1


class SimpleRNG:
    """simpleRNG, optics/fft_test.go:63-68: 64-bit LCG -> uniform in [-0.5, 0.5)."""

    def __init__(self, seed: int):
        self.seed = seed & MASK64

    def next(self) -> float:
        self.seed = (self.seed * 6364136223846793005 + 1442695040888963407) & MASK64
        return float(self.seed >> 11) / 9007199254740992.0 - 0.5

    def complex_array(self, shape) -> np.ndarray:
        n = int(np.prod(shape))
        out = np.empty(n, dtype=np.complex128)
        for k in range(n):
            re = self.next()
            im = self.next()
            out[k] = complex(re, im)
        return out.reshape(shape)


def lcg_complex(seed: int, n: int) -> np.ndarray:
    """Vectorised SimpleRNG stream (same values as SimpleRNG.complex_array)."""
    a, c = 6364136223846793005, 1442695040888963407
    vals = np.empty(2 * n, dtype=np.float64)
    s = seed & MASK64
    # block-wise jump: s_{k+1} = a s_k + c  (mod 2^64), using python ints in chunks
    for k in range(2 * n):
        s = (s * a + c) & MASK64
        vals[k] = float(s >> 11) / 9007199254740992.0 - 0.5
    return vals[0::2] + 1j * vals[1::2]


def ref_field(n: int, seed: float) -> np.ndarray:
    """refField, optics/gpu_test.go:12-22."""
    i = np.arange(n, dtype=np.float64)[None, :]
    j = np.arange(n, dtype=np.float64)[:, None]
    ii = np.arange(n)[None, :]
    jj = np.arange(n)[:, None]
    re = np.sin(seed * (i + 1) * 0.7) + 0.5 * np.cos(seed * (j + 1))
    im = np.cos(seed * (ii - jj).astype(np.float64) * 0.3) - 0.25 * np.sin(seed * (ii * jj + 1).astype(np.float64))
    return re + 1j * im


def naive_dft(a: np.ndarray) -> np.ndarray:
    """naiveDFT1D, optics/asm_improve_test.go:10-21."""
    n = a.size
    k = np.arange(n)
    w = np.exp(-2j * np.pi * np.outer(k, k) / n)
    return w @ a


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """relCmpL2, optics/complex_field_test.go:15-26 (and relL2, asm_accuracy_test.go:34-46)."""
    num = np.sum(np.abs(a - b) ** 2)
    den = np.sum(np.abs(b) ** 2)
    return 0.0 if den <= 0 else float(np.sqrt(num / den))


def centroid_x(f) -> float:
    """centroidX, optics/asm_accuracy_test.go:19-32."""
    w = f.intensity()
    x = f.x(np.arange(f.nx))
    p = w.sum()
    return 0.0 if p <= 0 else float((w * x[None, :]).sum() / p)


def waist_radius(f) -> float:
    """waistRadius, optics/volume_test.go:35-46."""
    w = f.intensity()
    x = f.x(np.arange(f.nx))[None, :]
    y = f.y(np.arange(f.ny))[:, None]
    return float(np.sqrt(2 * (w * (x * x + y * y)).sum() / w.sum()))


def evanescent_field(n: int, dx: float, q: int) -> np.ndarray:
    """evanescentField, optics/asm_improve_test.go:169-178."""
    f0 = q / (n * dx)
    x = (np.arange(n) - n / 2) * dx
    row = np.exp(1j * 2 * np.pi * f0 * x)
    return np.tile(row, (n, 1))


def single_bin_plane_wave(n: int, dx: float, wl: float, sx: float, sy: float) -> np.ndarray:
    """singleBinTiltedPlaneWave, optics/complex_field_test.go:32-42."""
    k = 2 * math.pi / wl
    x = (np.arange(n) - n / 2) * dx
    y = (np.arange(n) - n / 2) * dx
    return np.exp(1j * k * (sx * x[None, :] + sy * y[:, None]))


def analytic_gaussian_fresnel(n: int, dx: float, wl: float, z: float, w0: float) -> np.ndarray:
    """analyticGaussianFresnel, optics/complex_field_test.go:90-111."""
    beta = complex(1 / (w0 * w0), -math.pi / (wl * z))
    x = (np.arange(n) - n / 2) * dx
    gamma = 2 * math.pi * x / (wl * z)
    G = np.sqrt(math.pi / beta) * np.exp(1j * math.pi * x * x / (wl * z)) * np.exp(-gamma * gamma / (4 * beta))
    pre = np.exp(1j * 2 * math.pi / wl * z) / complex(0, wl * z)
    return pre * G[:, None] * G[None, :]


def far_field_radius(I: np.ndarray, n: int, dx_out: float) -> float:
    """farFieldRadius, optics/coherence_test.go:69-126."""
    nbins = 128
    s = np.zeros(nbins)
    cnt = np.zeros(nbins)
    max_r = dx_out * n / 2
    dr = max_r / nbins
    x = (np.arange(n) - n / 2) * dx_out
    r = np.hypot(x[None, :], x[:, None])
    b = (r / dr).astype(np.int64)
    m = b < nbins
    np.add.at(s, b[m], I[m])
    np.add.at(cnt, b[m], 1)
    ok = cnt > 0
    v = np.where(ok, s / np.maximum(cnt, 1), 0)
    peak = v[ok].max()
    sel = ok & (v >= 0.02 * peak)
    rr = (np.arange(nbins) + 0.5) * dr
    r2 = rr * rr
    w = cnt
    lv = np.log(np.where(sel, v, 1))
    sw = (w * sel).sum(); sx = (w * r2 * sel).sum(); sy = (w * lv * sel).sum()
    sxx = (w * r2 * r2 * sel).sum(); sxy = (w * r2 * lv * sel).sum()
    den = sw * sxx - sx * sx
    if sw < 4 or den == 0:
        return 0.0
    c = (sw * sxy - sx * sy) / den
    if c >= 0:
        return 0.0
    return math.sqrt(-2 / c)


# --------------------------------------------------------------------------
# Harness noise: splitmix64 + Box-Muller.  The reference draws the Schell
# noise from Go's math/rand (coherence.go:63-70), which is not vendored in the
# reference tree; this seeded generator stands in for it and feeds identical
# values to the oracle and to the GPU path.
# --------------------------------------------------------------------------
def splitmix64(seed: int, count: int) -> np.ndarray:
    out = np.empty(count, dtype=np.uint64)
    with np.errstate(over="ignore"):
        idx = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    out[:] = z
    return out


def uniform01(seed: int, count: int) -> np.ndarray:
    return (splitmix64(seed, count) >> np.uint64(11)).astype(np.float64) / float(1 << 53)


def complex_normal(seed: int, shape) -> np.ndarray:
    """complex(N(0,1)/sqrt2, N(0,1)/sqrt2) values, Box-Muller on splitmix64 uniforms."""
    n = int(np.prod(shape))
    u = uniform01(seed, 2 * n)
    u1 = np.maximum(u[0::2], 1e-300)
    u2 = u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    re = r * np.cos(2 * np.pi * u2)
    im = r * np.sin(2 * np.pi * u2)
    return ((re + 1j * im) / math.sqrt(2)).reshape(shape)
