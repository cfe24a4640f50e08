"""The sharded batch entry points on the real backend over NCCL: one rank on
one GPU (this pool gives one GPU per run; the multi-rank logic is covered on
CPU with gloo in test_shard.py).  The all-reduce / all-gather then run through
NCCL on CUDA tensors and must return the unsharded results."""
import importlib
import os
import socket

import numpy as np
import pytest

from gpu_util import wos

pytestmark = pytest.mark.gpu


def _worker(rank, port, result_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1)
    shard = importlib.import_module("tetsuhiro-wos_b200.shard")
    try:
        g = wos.GPU(wos.FP32)
        rng = np.random.default_rng(1)
        n, dx = 256, 2e-6
        ex = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        wls, wts = [500e-9, 600e-9, 700e-9], [1.0, 0.5, 0.25]
        want = g.polychromatic(wos.Field(ex.copy(), dx), 2e-3, wls, wts, "asm", wos.Context(wavelength=6e-7))
        got = shard.polychromatic_sharded(g, wos.Field(ex.copy(), dx), 2e-3, wls, wts, "asm",
                                          wos.Context(wavelength=6e-7))
        assert np.array_equal(got, want)
        zs = [0.0, 1e-3, 3e-3]
        vw = g.volume(wos.Field(ex.copy(), dx), zs, "asm", wos.Context(wavelength=6e-7))
        vg = shard.volume_sharded(g, wos.Field(ex.copy(), dx), zs, "asm", wos.Context(wavelength=6e-7))
        assert np.array_equal(vg, vw)
        g.close()
        open(os.path.join(result_dir, "ok"), "w").close()
    finally:
        dist.destroy_process_group()


def test_sharded_units_over_nccl_one_rank(tmp_path):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_worker, args=(port, str(tmp_path)), nprocs=1, join=True)
    assert (tmp_path / "ok").exists()
