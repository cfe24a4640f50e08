"""The sharded device batches through the C ABI (wos_comm_init and the
*_sharded_dev calls) on a one-rank communicator, the only one a single GPU
allows: each must return exactly what the unsharded device call returns.
The split itself (wos_shard_range) and the exchange step are covered with
two and three gloo ranks on the CPU (tests/test_shard.py)."""
import importlib

import numpy as np
import pytest
import torch

from gpu_util import wos

W = importlib.import_module("tetsuhiro-wos_b200.workloads")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [wos.FP64, wos.FP32], ids=["fp64", "fp32"])
def test_one_rank_sharded_batches_equal_the_unsharded_calls(prec):
    dt = torch.complex128 if prec == wos.FP64 else torch.complex64
    d1, d2, d3 = W.cfg4_1(), W.cfg4_2(12), W.cfg4_3(10)
    n1, n2, n3 = d1["ex"].shape[0] // 4, d2["n"] // 2, d3["ex"].shape[0] // 2
    ex1 = d1["ex"][:n1, :n1].copy()
    ex3 = d3["ex"][::2, ::2].copy()
    noise = d2["noise"][:, :n2, :n2].copy()
    with wos.GPU(prec) as g:
        g.comm_init(1, 0, wos.comm_unique_id())
        f1 = torch.from_numpy(ex1[None]).to(dt).cuda()
        f3 = torch.from_numpy(ex3[None]).to(dt).cuda()
        nz = torch.from_numpy(noise).cuda()
        outs = []
        for sharded in (False, True):
            o1 = torch.empty((n1, n1), dtype=torch.float64, device="cuda")
            o2 = torch.empty((n2, n2), dtype=torch.float64, device="cuda")
            o3 = torch.empty((d3["zs"].size, 1, n3, n3), dtype=dt, device="cuda")
            torch.cuda.synchronize()
            c1, c2 = wos.Context(wavelength=d1["wls"][0]), wos.Context(wavelength=d2["wl"])
            c3 = wos.Context(wavelength=d3["wl"])
            if sharded:
                g.polychromatic_sharded_dev(n1, n1, d1["dx"], 1, f1.data_ptr(), d1["z"], d1["wls"], d1["weights"], c1,
                                            o1.data_ptr())
                g.partially_coherent_sharded_dev(n2, d2["dx"], d2["width"], d2["coherence"], 12, nz.data_ptr(),
                                                 d2["z"], c2, o2.data_ptr())
                g.volume_sharded_dev(n3, n3, d3["dx"], 1, f3.data_ptr(), d3["zs"], c3, o3.data_ptr())
            else:
                g.polychromatic_dev(n1, n1, d1["dx"], 1, f1.data_ptr(), d1["z"], d1["wls"], d1["weights"], c1,
                                    o1.data_ptr())
                g.partially_coherent_dev(n2, d2["dx"], d2["width"], d2["coherence"], 12, nz.data_ptr(), d2["z"], c2,
                                         o2.data_ptr())
                g.volume_dev(n3, n3, d3["dx"], 1, f3.data_ptr(), d3["zs"], c3, o3.data_ptr())
            g.synchronize()
            outs.append([o.cpu().numpy() for o in (o1, o2, o3)])
        g.comm_destroy()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_sharded_call_without_communicator_is_rejected():
    with wos.GPU(wos.FP32) as g:
        out = torch.empty((8, 8), dtype=torch.float64, device="cuda")
        f = torch.zeros((1, 8, 8), dtype=torch.complex64, device="cuda")
        with pytest.raises(wos.WosError) as e:
            g.polychromatic_sharded_dev(8, 8, 1e-6, 1, f.data_ptr(), 1e-3, [5e-7], [1.0],
                                        wos.Context(wavelength=5e-7), out.data_ptr())
        assert e.value.status == 6   # WOS_NOT_INITIALISED
