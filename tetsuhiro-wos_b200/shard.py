"""Batched units sharded over the ranks of a torch.distributed group (one
process per GPU).

The batch entry points of the reference loop over independent units:
wavelengths (PropagatePolychromatic, optics/polychromatic.go:18-44), coherent
modes (PropagatePartiallyCoherent, optics/coherence.go:105-116) and distances
(Propagate3D, optics/volume.go:8-18).  Each rank takes a contiguous range of
the units and runs it through its own context (wos_polychromatic /
wos_partially_coherent / wos_volume); the only data exchange is one FP64
all-reduce of the intensity map (polychromatic, partially coherent) or one
all-gather of the planes (volume), over NCCL between GPUs (gloo on CPU).  A
single propagation is not sharded: its 2-D FFT would need an all-to-all
transpose per sweep, which costs more than the whole step on one GPU.

Warnings: each rank's context collects the warnings of its own units; the
merged set is what the sequential loop would have added to the shared
ctx.Warnings (counts summed, the last unit's value kept), in unit order.
"""
from __future__ import annotations

from typing import List, Optional, Tuple

import numpy as np


def unit_range(n_units: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous, balanced [lo, hi) of the units rank `rank` runs: the first
    n_units % world ranks take one unit more."""
    base, extra = divmod(n_units, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _dist(group):
    import torch.distributed as dist
    return dist, dist.get_rank(group), dist.get_world_size(group)


def _all_reduce_sum(arr: np.ndarray, group) -> np.ndarray:
    import torch
    dist, _, _ = _dist(group)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float64)).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def _all_gather_rows(arr: np.ndarray, counts: List[int], group) -> np.ndarray:
    """Concatenate every rank's leading-axis block (rank order)."""
    import torch
    dist, rank, world = _dist(group)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    per = arr.shape[1:]
    mx = max(counts)
    pad = np.zeros((mx,) + per, dtype=arr.dtype)
    pad[: arr.shape[0]] = arr
    t = torch.from_numpy(pad.view(np.float64)).to(dev)  # complex128 travels as float64 pairs
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t, group=group)
    parts = [o.cpu().numpy().view(arr.dtype)[:c] for o, c in zip(outs, counts)]
    return np.concatenate(parts, axis=0)


def _merge_warnings(ctx, group) -> None:
    """Replace ctx.warnings on every rank by the merge, in rank (unit) order."""
    if ctx is None or not getattr(ctx, "warnings_enabled", True):
        return
    dist, _, world = _dist(group)
    allw = [None] * world
    dist.all_gather_object(allw, dict(ctx.warnings), group=group)
    merged = {}
    for w in allw:
        for code, (cnt, val) in w.items():
            c0, v0 = merged.get(code, (0, 0.0))
            merged[code] = (c0 + cnt, val if val != 0 else v0)
    ctx.warnings.clear()
    ctx.warnings.update(merged)


def polychromatic_sharded(gpu, f, z: float, wavelengths, weights, method: str = "asm", ctx=None,
                          group=None) -> np.ndarray:
    """PropagatePolychromatic with the wavelengths split over the ranks; every
    rank returns the full weighted intensity sum (float64 (ny, nx))."""
    wl = np.asarray(wavelengths, dtype=np.float64)
    w = np.asarray(weights, dtype=np.float64)
    if wl.size == 0:
        raise ValueError("polychromatic: no wavelength samples")
    if np.any(wl <= 0):
        raise ValueError("polychromatic: wavelengths must be > 0")
    _, rank, world = _dist(group)
    lo, hi = unit_range(wl.size, rank, world)
    part = np.zeros((f.ny, f.nx))
    if hi > lo:
        part = gpu.polychromatic(f, z, wl[lo:hi], w[lo:hi], method, ctx)
    out = _all_reduce_sum(part, group)
    _merge_warnings(ctx, group)
    return out


def partially_coherent_sharded(gpu, n: int, dx: float, width: float, coherence: float, noise: np.ndarray,
                               z: float, method: str = "asm", ctx=None, group=None) -> np.ndarray:
    """PropagatePartiallyCoherent with the modes split over the ranks: each rank
    averages its modes, the averages are combined with weights m_rank / m."""
    m = noise.shape[0]
    if m == 0:
        raise ValueError("partially coherent: no modes")
    _, rank, world = _dist(group)
    lo, hi = unit_range(m, rank, world)
    part = np.zeros((n, n))
    if hi > lo:
        part = gpu.partially_coherent(n, dx, width, coherence, noise[lo:hi], z, method, ctx) * ((hi - lo) / m)
    out = _all_reduce_sum(part, group)
    _merge_warnings(ctx, group)
    return out


def volume_sharded(gpu, f, zs, method: str = "asm", ctx=None, group=None) -> np.ndarray:
    """Propagate3D with the distances split over the ranks; every rank returns
    the whole volume (nz, ncomp, ny, nx) complex128, planes in zs order."""
    z = np.asarray(zs, dtype=np.float64)
    _, rank, world = _dist(group)
    counts = [unit_range(z.size, r, world)[1] - unit_range(z.size, r, world)[0] for r in range(world)]
    lo, hi = unit_range(z.size, rank, world)
    ncomp = 2 if f.polarized else 1
    part = np.zeros((hi - lo, ncomp, f.ny, f.nx), dtype=np.complex128)
    if hi > lo:
        part = gpu.volume(f, z[lo:hi], method, ctx)
    out = _all_gather_rows(part, counts, group)
    _merge_warnings(ctx, group)
    return out
