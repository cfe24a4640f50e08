"""Sharded batch units (tetsuhiro-wos_b200/shard.py) on CPU: two gloo ranks,
each running its contiguous range of units through a stand-in backend that
computes with the oracle, must reproduce the single-process oracle results
(intensity maps to 1e-13, planes exactly, warnings merged in unit order)."""
import importlib
import os
import socket

import numpy as np
import pytest

import oracle as O

shard = importlib.import_module("tetsuhiro-wos_b200.shard")


def test_unit_ranges_cover_every_unit_once():
    for n in range(0, 13):
        for world in range(1, 6):
            got = [shard.unit_range(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [hi - lo for lo, hi in got]
            assert max(sizes) - min(sizes) <= 1


class OracleUnits:
    """The batch entry points of the GPU binding, computed with the oracle."""

    def polychromatic(self, f, z, wls, weights, method, ctx):
        return O.polychromatic(O.Field(f.ex.copy(), f.dx, f.ey.copy() if f.polarized else None), z, wls, weights,
                               method, ctx)

    def volume(self, f, zs, method, ctx):
        return O.propagate3d(O.Field(f.ex.copy(), f.dx, f.ey.copy() if f.polarized else None), zs, method, ctx)

    def partially_coherent(self, n, dx, width, coherence, noise, z, method, ctx):
        modes = O.schell_realizations(n, dx, width, coherence, noise)
        for k in range(modes.shape[0]):
            f = O.Field(modes[k].copy(), dx)
            O.propagate(f, z, method, ctx)
            modes[k] = f.ex
        return O.average_intensity(modes)


def _case():
    rng = np.random.default_rng(3)
    n, dx = 32, 2e-6
    ex = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    noise = (rng.normal(size=(5, n, n)) + 1j * rng.normal(size=(5, n, n))) / np.sqrt(2)
    return n, dx, ex, noise


def _reference():
    n, dx, ex, noise = _case()
    wls, wts, zs = [500e-9, 550e-9, 600e-9, 650e-9, 700e-9], [1, 0.8, 0.6, 0.4, 0.2], [0.0, 1e-3, 2e-3, 4e-3, 8e-3]
    u = OracleUnits()
    c1 = O.Context(wavelength=600e-9)
    poly = u.polychromatic(O.Field(ex.copy(), dx), 5e-3, wls, wts, "asm", c1)
    c2 = O.Context(wavelength=600e-9)
    vol = u.volume(O.Field(ex.copy(), dx), zs, "asm", c2)
    c3 = O.Context(wavelength=633e-9)
    pc = u.partially_coherent(n, dx, 40e-6, 8e-6, noise, 3e-3, "asm", c3)
    return (poly, dict(c1.warnings)), (vol, dict(c2.warnings)), (pc, dict(c3.warnings)), (wls, wts, zs)


def _worker(rank, world, port, result_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n, dx, ex, noise = _case()
        (poly, w1), (vol, w2), (pc, w3), (wls, wts, zs) = _reference()
        u = OracleUnits()
        c1 = O.Context(wavelength=600e-9)
        got = shard.polychromatic_sharded(u, O.Field(ex.copy(), dx), 5e-3, wls, wts, "asm", c1)
        assert np.max(np.abs(got - poly)) <= 1e-13 * np.max(np.abs(poly))
        assert c1.warnings == w1, (c1.warnings, w1)
        c2 = O.Context(wavelength=600e-9)
        gv = shard.volume_sharded(u, O.Field(ex.copy(), dx), zs, "asm", c2)
        assert gv.shape == vol.shape and np.array_equal(gv, vol)
        assert c2.warnings == w2
        c3 = O.Context(wavelength=633e-9)
        gp = shard.partially_coherent_sharded(u, n, dx, 40e-6, 8e-6, noise, 3e-3, "asm", c3)
        assert np.max(np.abs(gp - pc)) <= 1e-13 * np.max(np.abs(pc))
        assert c3.warnings == w3
        open(os.path.join(result_dir, f"ok{rank}"), "w").close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_units_match_single_process(tmp_path, world):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True)
    assert all((tmp_path / f"ok{r}").exists() for r in range(world))


def test_c_abi_shard_range_matches_the_python_partition():
    """wos_shard_range (the partition of the C-ABI sharded batches, host only)
    is the same contiguous split as shard.unit_range, which the gloo tests
    above run end to end; invalid arguments are rejected."""
    wos = importlib.import_module("tetsuhiro-wos_b200")
    for n in range(0, 40):
        for world in range(1, 9):
            for r in range(world):
                assert wos.shard_range(n, world, r) == shard.unit_range(n, r, world)
    for bad in ((4, 0, 0), (4, 2, 2), (-1, 2, 0), (4, 2, -1)):
        with pytest.raises(wos.WosError):
            wos.shard_range(*bad)
