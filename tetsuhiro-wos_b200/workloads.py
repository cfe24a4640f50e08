"""Seeded synthetic inputs of the propagation workloads, shared by bench.py and
the tests so that both measure and check the same fields.

No dataset is involved: each workload is the optical set-up named in its
docstring, built from seeded numpy generators.  Every function returns plain
numpy arrays and numbers (index-medium and context parameters as keyword
dicts), so the caller can hand them to the library or to the oracle alike.
"""
from __future__ import annotations

import numpy as np


def coords(n: int, dx: float) -> np.ndarray:
    """Centred pixel coordinates x(i) = (i - n/2) dx (optics/field.go:59-62)."""
    return (np.arange(n, dtype=np.float64) - n / 2) * dx


def random_phase(n: int, seed: int = 1) -> np.ndarray:
    """Unit amplitude, phase uniform in [0, 2 pi): excites every frequency bin."""
    rng = np.random.default_rng(seed)
    return np.exp(1j * rng.uniform(0, 2 * np.pi, (n, n))).astype(np.complex128)


def lens_beam(n: int, dx: float = 2e-6, wl: float = 632.8e-9, waist: float = 200e-6, radius: float = 400e-6,
              focal: float = 0.2) -> np.ndarray:
    """Gaussian beam exp(-r^2/w^2) clipped by a circular aperture of the given
    radius and multiplied by the thin-lens phase exp(-i pi r^2 / (wl f))."""
    x = coords(n, dx)
    r2 = x[None, :] ** 2 + x[:, None] ** 2
    ex = np.exp(-r2 / waist ** 2) * np.exp(-1j * np.pi * r2 / (wl * focal))
    ex[r2 > radius ** 2] = 0
    return ex.astype(np.complex128)


# --------------------------------------------------------------- single ASM
HEADLINE = dict(n=2048, dx=2e-6, wl=632.8e-9, z=0.05, method="asm")


def cfg1():
    """512^2 plain band-limited ASM, complex128: lens beam, z = 5 cm,
    Evanescent "zero"."""
    n, dx, wl = 512, 2e-6, 632.8e-9
    return dict(ex=lens_beam(n, dx, wl), ey=None, dx=dx, wl=wl, z=0.05, method="asm", evanescent="zero")


def cfg2():
    """1000 x 1500 asm_shift_pad with two Jones components: Ex a unit plane
    wave with a seeded diffuser phase uniform in [0, 2 pi) per 4 x 4-pixel
    cell, tilted by 3 degrees along x; Ey = 0.5 i Ex.  dx = 1 um,
    wl = 532 nm, z = 2 mm."""
    rng = np.random.default_rng(1)
    ny, nx, dx, wl, z = 1000, 1500, 1e-6, 532e-9, 2e-3
    cells = rng.uniform(0, 1, ((ny + 3) // 4, (nx + 3) // 4))
    u = np.repeat(np.repeat(cells, 4, axis=0), 4, axis=1)[:ny, :nx]
    x = coords(nx, dx)
    ex = np.exp(2j * np.pi * u) * np.exp(1j * 2 * np.pi / wl * np.sin(np.radians(3)) * x)[None, :]
    return dict(ex=ex.astype(np.complex128), ey=(0.5j * ex).astype(np.complex128), dx=dx, wl=wl, z=z,
                method="asm_shift_pad", evanescent="decay")


# --------------------------------------------------------------- split-step
def cfg3(slices: int = 400):
    """Split-step BPM: 1024^2, dx = 0.5 um, wl = 1.55 um, `slices` slices of
    dz = 2 um through n = 1.45 + 0.01 exp(-r^2/(25 um)^2) (1 + 0.1 sin(2 pi z
    / 200 um)) + 1e-5 i, plus an absorbing border 32 px wide (Im n +=
    5e-3 ((32 - d)/32)^2 at edge distance d < 32).  Input: Gaussian of waist
    8 um centred at x = +5 um."""
    n, dx, wl, dz = 1024, 0.5e-6, 1.55e-6, 2e-6
    x = coords(n, dx)
    ex = np.exp(-((x[None, :] - 5e-6) ** 2 + x[:, None] ** 2) / (8e-6) ** 2).astype(np.complex128)
    desc = dict(re_bg=1.45, im_bg=1e-5, core_dn=0.01, core_w=25e-6, zmod_amp=0.1, zmod_period=200e-6,
                border_px=32, border_order=2, border_strength=5e-3)
    return dict(ex=ex, dx=dx, wl=wl, z=slices * dz, steps=slices, desc=desc)


def index_desc(cls, params: dict):
    """An IndexDesc (library's or oracle's class) from a parameter dict."""
    d = cls()
    for k, v in params.items():
        setattr(d, k, v)
    return d


# --------------------------------------------------------------- batches
def cfg4_1():
    """Polychromatic ASM: 64 wavelengths uniform over 400-700 nm (weights 1),
    1024^2, dx = 2 um, z = 1 cm, a plane wave through an amplitude-binary
    grating of period 20 um and duty 0.5 (t = 1 iff cos(2 pi x / period) >=
    cos(pi duty), optics/elements.go:496-499)."""
    n, dx, z = 1024, 2e-6, 0.01
    x = coords(n, dx)
    t = (np.cos(2 * np.pi * x / 20e-6) >= np.cos(np.pi * 0.5)).astype(np.float64)
    ex = np.repeat(t[None, :], n, axis=0).astype(np.complex128)
    wls = np.linspace(400e-9, 700e-9, 64)
    return dict(ex=ex, dx=dx, z=z, wls=wls, weights=np.ones(64))


def cfg4_2(modes: int = 256):
    """Gaussian Schell source: `modes` coherent modes on 512^2, dx = 4 um,
    intensity width w0 = 600 um (exp(-2 r^2 / w0^2)), coherence length 50 um,
    z = 1 cm, wl = 632.8 nm; the complex normal noise of each mode (the
    place of Go's math/rand draws, optics/coherence.go:63-70) is seeded."""
    n, dx = 512, 4e-6
    rng = np.random.default_rng(1)
    noise = (rng.standard_normal((modes, n, n)) + 1j * rng.standard_normal((modes, n, n))) / np.sqrt(2)
    return dict(n=n, dx=dx, width=600e-6, coherence=50e-6, noise=noise, z=0.01, wl=632.8e-9)


def cfg4_3(planes: int = 128):
    """3-D volume: `planes` distances evenly over 0-10 mm (z = 0 returns the
    input), 768^2, dx = 4 um, Gaussian of waist 300 um, wl = 632.8 nm."""
    n, dx, wl = 768, 4e-6, 632.8e-9
    x = coords(n, dx)
    ex = np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / (300e-6) ** 2).astype(np.complex128)
    return dict(ex=ex, dx=dx, wl=wl, zs=np.linspace(0, 0.01, planes))


# --------------------------------------------------------------- inverse design
def spots_target(n: int, dx: float, rng, count: int = 16, sigma: float = 20e-6) -> np.ndarray:
    """Sum of `count` Gaussian spots exp(-r^2 / (2 sigma^2)) at positions
    uniform in the central 60 % of the window."""
    x = coords(n, dx)
    t = np.zeros((n, n))
    for cx, cy in rng.uniform(-0.3, 0.3, (count, 2)) * n * dx:
        t += np.exp(-((x[None, :] - cx) ** 2 + (x[:, None] - cy) ** 2) / (2 * sigma ** 2))
    return t


def cfg5():
    """Phase-only mask design: 2048^2, dx = 4 um, wl = 633 nm, z = 10 cm,
    plane-wave illumination, phi uniform in [0, 2 pi) (seed 1), target 16
    Gaussian spots (sigma 20 um)."""
    n, dx = 2048, 4e-6
    rng = np.random.default_rng(1)
    phi = rng.uniform(0, 2 * np.pi, (n, n))
    tgt = spots_target(n, dx, rng)
    return dict(a=np.ones((n, n), dtype=np.complex128), phi=phi, target=tgt, dx=dx, wl=633e-9, z=0.1)


def cfg5_2(layers: int = 3, slices: int = 200):
    """Diffractive stack: `layers` phase masks on 2048^2 (dx = 4 um, wl =
    633 nm), each followed by `slices` BPM slices of 5 um through a uniform
    n = 1.5 medium; plane-wave illumination, target 16 Gaussian spots."""
    n, dx = 2048, 4e-6
    rng = np.random.default_rng(1)
    phis = rng.uniform(0, 2 * np.pi, (layers, n, n))
    tgt = spots_target(n, dx, rng)
    return dict(a=np.ones((n, n), dtype=np.complex128), phis=phis, target=tgt, dx=dx, wl=633e-9,
                zseg=slices * 5e-6, steps=slices, desc=dict(re_bg=1.5))
