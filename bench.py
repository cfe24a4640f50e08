#!/usr/bin/env python3
"""Headline benchmark: 2048^2 scalar band-limited ASM propagations per second.

Workload (one "step" = --batch propagations of distinct fields, 1536 by default):
  2048 x 2048 grid, dx = 2 um, lambda = 632.8 nm, z = 5 cm, complex64 pipeline
  (FP64 transfer-function argument), device-resident fields propagated in place
  through the C ABI: wos_propagate_batch_dev calls of up to 64 fields over a
  pool of 64 distinct 32 MiB fields (2 GiB working set, > 16x the 126 MB L2),
  which run the independent fields on two streams; the rate of one
  wos_propagate_dev call per field is reported beside it.  Inputs: a seeded
  unit-amplitude random-phase field (excites every frequency bin).  Both arms
  use the same Context: Warnings nil (the reference's default Context), so
  neither runs the alias-wrap check nor the power sums.
Also reported: the FP64 (complex128) kernel on the same workload, the
end-to-end rate through the host API (complex128 host buffers, H2D + D2H in
the timed region; page-locked and pageable), the roofline of the dominant
kernel from live per-launch CUDA events, the FP32 and FP64 results against
the FP64 oracle on the same input, and the oracle's CPU rate on this host.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: replicas (one independent propagation stream per rank); value is
the job-wide rate = all ranks' propagations / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
WL_ = importlib.import_module("tetsuhiro-wos_b200.workloads")

METRIC = "2048² ASM props/s, FP32 vs FP64 GPU at rel-L2≤1e-5; % HBM roofline"
N = 2048
DX = 2e-6
WL = 632.8e-9
ZPROP = 0.05
POOL = 64


BATCH = 1536


def workload_config() -> dict:
    return {"workload": f"asm {N}x{N} scalar, complex64, dx=2um, lambda=632.8nm, z=5cm",
            "grid": [N, N], "method": "asm", "evanescent": "decay",
            "warnings": "off: ctx.Warnings nil (the reference default), no wrap check or power sums",
            "input": "unit-amplitude random phase (seed 1); the lens recipe is timed and checked beside it "
                     "(lens_input)",
            "l2_flush": f"inputs larger than L2: {POOL} distinct {N * N * 8 >> 20} MiB fields in rotation",
            "parallelism": "replicas"}


def measured_peaks() -> tuple:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def input_field(seed: int = 1) -> np.ndarray:
    return WL_.random_phase(N, seed)


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def oracle_context(O):
    """The Context of both arms: Warnings nil (optics.Propagate's default)."""
    return O.Context(wavelength=WL, warnings_enabled=False)


def cpu_baseline(ex: np.ndarray, sample_props: int = 3):
    """The FP64 oracle (C restatement of the reference's Go CPU path) on this
    host: its rate, and its output field (the parity reference of the run)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # noqa: E402  (CPU-baseline leg only)
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    t_total = 0.0
    done = 0
    out = None
    for _ in range(sample_props):
        f = O.Field(ex.copy(), DX)
        t0 = time.perf_counter()
        O.propagate(f, ZPROP, "asm", oracle_context(O))
        t_total += time.perf_counter() - t0
        done += 1
        out = f.ex
        if t_total > 30:
            break
    return {"value": done / t_total, "unit": "props/s", "cores": cores, "kind": "port",
            "sample": f"{done} propagation(s) of the {N}x{N} workload, FP64 C oracle, {cores} threads "
                      "(parFor semantics of optics/fft.go:91-122), the same Context as the GPU arm",
            "seconds": t_total}, out


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # noqa: E402  (reference arm: the reference algorithm on the host cores)
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    ex = input_field()
    for _ in range(args.warmup):
        f = O.Field(ex.copy(), DX)
        O.propagate(f, ZPROP, "asm", oracle_context(O))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        f = O.Field(ex.copy(), DX)
        O.propagate(f, ZPROP, "asm", oracle_context(O))
    dt = time.perf_counter() - t0
    v = args.steps / dt
    line = {"metric": METRIC, "value": v, "unit": "props/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": workload_config(), "fields_per_step": 1,
            "cpu_baseline": {"value": v, "unit": "props/s", "cores": cores, "kind": "port",
                             "sample": f"one {N}x{N} propagation per step, FP64 C oracle "
                                       "(restatement of optics/fft.go + optics/propagate.go), "
                                       f"{cores} threads"},
            "e2e": {"value": v, "unit": "props/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def time_batch(g, torch, bufs, steps, warmup, batch, ctx, stream):
    """Device-resident timed region: `batch` propagations per step, issued as
    wos_propagate_batch_dev calls of up to len(bufs) fields over the pool."""
    ptrs = [b.data_ptr() for b in bufs]
    chunks, left = [], batch
    while left > 0:
        k = min(left, len(ptrs))
        chunks.append(ptrs[:k])
        left -= k

    def step():
        for c in chunks:
            g.propagate_batch_dev(N, N, DX, 1, c, c, ZPROP, "asm", ctx)
    for _ in range(warmup):
        step()
    launches0 = g.launch_count()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), g.launch_count() - launches0


def time_device(g, torch, bufs, steps, warmup, batch, ctx, stream, profile=False):
    """Device-resident timed region: steps x batch in-place propagations."""
    n = 0
    for _ in range(warmup * batch):
        b = bufs[n % len(bufs)]
        g.propagate_dev(N, N, DX, 1, b.data_ptr(), b.data_ptr(), ZPROP, "asm", ctx)
        n += 1
    if profile:
        g.synchronize()
        g.profile_reset()
        g.set_profiling(True)
    launches0 = g.launch_count()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps * batch):
        b = bufs[n % len(bufs)]
        g.propagate_dev(N, N, DX, 1, b.data_ptr(), b.data_ptr(), ZPROP, "asm", ctx)
        n += 1
    e1.record(stream)
    torch.cuda.synchronize()
    launches = g.launch_count() - launches0
    prof = g.profile() if profile else {}
    if profile:
        g.set_profiling(False)
    return e0.elapsed_time(e1), launches, prof



# ---------------------------------------------------------------------------
# Secondary configurations of the workload table (one JSON line each):
#   python bench.py --config {cfg1,cfg2,cfg3,cfg4.1,cfg4.2,cfg4.3,cfg5,cfg5.2,train}
# Seeded synthetic inputs of the stated shapes stand in for the reference's
# cases; timed through the library's public entry points with CUDA events on
# the context's stream (host-buffer entry points include their H2D/D2H, with
# page-locked host buffers where the entry point moves large arrays); a
# bounded sample of the FP64 oracle on the host cores gives the CPU figure.
def _cfg_inputs(name: str):
    return {"cfg1": WL_.cfg1, "cfg2": WL_.cfg2}[name]()


def _algorithmic_bytes(name: str, esz: int) -> float:
    """Per-run algorithmic bytes of the workload table (complex64: esz = 8)."""
    k = esz / 8
    return {"cfg1": 48 * 512 ** 2 * k, "cfg2": 2 * 104 * 1.5e6 * k, "cfg3": 803 * 16 * 1024 ** 2 * k,
            "cfg4.1": (32 + 64 * 32) * 1024 ** 2 * k, "cfg4.2": 256 * 56 * 512 ** 2 * k,
            "cfg4.3": 32 * 768 ** 2 * 129 * k, "cfg5": 108 * 2048 ** 2 * k,
            "cfg4": ((32 + 64 * 32) * 1024 ** 2 + 256 * 56 * 512 ** 2 + 32 * 768 ** 2 * 129) * k,
            # diffractive stack, 3 layers x 200 slices, forward + adjoint: 2 nl (2S + 3)
            # field sweeps (R+W) plus per-layer mask / state / gradient passes and the residual
            "cfg5.2": (2 * 3 * (2 * 200 + 3) * 16 + 3 * 72 + 24) * 2048 ** 2 * k,
            # element train: 3 elements on the complex128 planes (32 B/px each), 3
            # propagations (64 B/px each: complex128 in and out of the FP32 sweeps), one sensor
            "train": (3 * 32 + 3 * 64 + 24) * 2048 ** 2}[name]


def _graph_of(g, fn):
    """Capture the device-resident calls of fn (already run once) in a CUDA
    graph; None when a call inside needs a synchronisation."""
    g.synchronize()
    g.graph_capture_begin()
    try:
        fn()
    except Exception:
        pass
    try:
        return g.graph_capture_end()
    except Exception:
        return None


def run_config(args) -> None:
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # noqa: E402  (CPU-baseline leg only)
    wos = importlib.import_module("tetsuhiro-wos_b200")
    name = args.config
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    peak, peak_kind = measured_peaks()
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    lines = []

    def timed(fn, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / steps  # s per run

    def cpu(fn, budget=20.0):
        t0 = time.perf_counter()
        n = 0
        while True:
            fn()
            n += 1
            if time.perf_counter() - t0 > budget / 4 or n >= 3:
                break
        return (time.perf_counter() - t0) / n

    for prec, pname, esz in ((wos.FP32, "f32", 8), (wos.FP64, "f64", 16)):
        g = wos.GPU(prec)
        g.set_stream(stream.cuda_stream)
        rec = {"precision": pname}
        if name in ("cfg1", "cfg2"):
            d = _cfg_inputs(name)
            ex, ey = d["ex"], d.get("ey")
            ctxk = dict(wavelength=d["wl"], evanescent=d.get("evanescent", "decay"))
            ncomp = 1 if ey is None else 2
            dt = torch.complex128 if prec == wos.FP64 else torch.complex64
            with torch.cuda.stream(stream):
                dev = [torch.from_numpy(np.stack([ex] if ey is None else [ex, ey])).to(dt).cuda() for _ in range(8)]
            torch.cuda.synchronize()
            ny, nx = ex.shape
            cnt = [0]

            def dev_run():
                b = dev[cnt[0] % 8]
                cnt[0] += 1
                g.propagate_dev(ny, nx, d["dx"], ncomp, b.data_ptr(), b.data_ptr(), d["z"], d["method"],
                                wos.Context(warnings_enabled=False, **ctxk))
            rec["device_s"] = timed(dev_run, args.steps, args.warmup)
            gr = _graph_of(g, lambda: [dev_run() for _ in range(8)])
            if gr is not None:  # the same calls replayed from a CUDA graph (wos_graph_launch)
                rec["device_direct_s"] = rec["device_s"]
                rec["device_s"] = timed(gr.launch, max(2, args.steps // 8), args.warmup) / 8
                rec["device_api"] = "wos_propagate_dev calls replayed from a CUDA graph"
                gr.close()
            hf = wos.Field(ex.copy(), d["dx"], None if ey is None else ey.copy())
            rec["e2e_s"] = timed(lambda: g.propagate(hf, d["z"], d["method"], wos.Context(**ctxk)),
                                 max(3, args.steps // 5), 2)
            if prec == wos.FP64:
                rec_cpu = cpu(lambda: O.propagate(O.Field(ex.copy(), d["dx"], None if ey is None else ey.copy()),
                                                  d["z"], d["method"], O.Context(**ctxk)))
        elif name == "cfg3":
            w3 = WL_.cfg3()
            ex, dx, wl, slices = w3["ex"], w3["dx"], w3["wl"], w3["steps"]
            n, dz = ex.shape[0], w3["z"] / w3["steps"]
            desc = WL_.index_desc(wos.IndexDesc, w3["desc"])
            dt = torch.complex128 if prec == wos.FP64 else torch.complex64
            with torch.cuda.stream(stream):
                dev = torch.from_numpy(ex).to(dt).cuda()
            torch.cuda.synchronize()
            bpm = lambda: g.split_step_dev(n, n, dx, 1, dev.data_ptr(), slices * dz, desc, slices,  # noqa: E731
                                           wos.Context(wavelength=wl, warnings_enabled=False))
            rec["device_s"] = timed(bpm, max(2, args.steps // 10), 1)
            gr = _graph_of(g, bpm)
            if gr is not None:  # the 801 sweeps replayed from a CUDA graph (wos_graph_launch)
                rec["device_direct_s"] = rec["device_s"]
                rec["device_s"] = timed(gr.launch, max(2, args.steps // 10), 1)
                rec["device_api"] = "wos_splitstep_dev replayed from a CUDA graph"
                gr.close()
            hf = wos.Field(ex.copy(), dx)
            rec["e2e_s"] = timed(lambda: g.split_step(hf, slices * dz, desc, slices, wos.Context(wavelength=wl)), 2, 1)
            if prec == wos.FP64:
                od = WL_.index_desc(O.IndexDesc, w3["desc"])
                t0 = time.perf_counter()
                O.splitstep(O.Field(ex.copy(), dx), 20 * dz, od, 20, O.Context(wavelength=wl))
                rec_cpu = (time.perf_counter() - t0) * slices / 20  # 20 of 400 slices, scaled
        elif name == "cfg4.1":
            n, dx, z = 1024, 2e-6, 0.01
            x = (np.arange(n) - n / 2) * dx
            t = (np.cos(2 * np.pi * x / 20e-6) >= np.cos(np.pi * 0.5)).astype(np.float64)
            ex = np.repeat(t[None, :], n, axis=0).astype(np.complex128)
            wls = np.linspace(400e-9, 700e-9, 64)
            hf = wos.Field(torch.from_numpy(ex).pin_memory().numpy(), dx)
            pout = torch.zeros((n, n), dtype=torch.float64).pin_memory().numpy()
            rec["e2e_s"] = timed(lambda: g.polychromatic(hf, z, wls, np.ones(64), "asm", wos.Context(wavelength=wls[0]),
                                                         out=pout), max(2, args.steps // 10), 1)
            if prec == wos.FP64:
                t0 = time.perf_counter()
                O.polychromatic(O.Field(ex.copy(), dx), z, wls[:4], np.ones(4), "asm", O.Context(wavelength=wls[0]))
                rec_cpu = (time.perf_counter() - t0) * 16  # 4 of 64 wavelengths, scaled
        elif name == "cfg4":
            # the three cfg4 parts on device buffers, recorded in one CUDA graph
            d1, d2, d3 = WL_.cfg4_1(), WL_.cfg4_2(), WL_.cfg4_3()
            n1, n2, n3 = d1["ex"].shape[0], d2["n"], d3["ex"].shape[0]
            m2 = d2["noise"].shape[0]
            dt = torch.complex128 if prec == wos.FP64 else torch.complex64
            with torch.cuda.stream(stream):
                f1 = torch.from_numpy(d1["ex"][None]).to(dt).cuda()
                f3 = torch.from_numpy(d3["ex"][None]).to(dt).cuda()
                nz = torch.from_numpy(d2["noise"]).cuda()
                o1 = torch.empty((n1, n1), dtype=torch.float64, device="cuda")
                o2 = torch.empty((n2, n2), dtype=torch.float64, device="cuda")
                o3 = torch.empty((d3["zs"].size, 1, n3, n3), dtype=dt, device="cuda")
            torch.cuda.synchronize()

            def part1(gx=g):
                gx.polychromatic_dev(n1, n1, d1["dx"], 1, f1.data_ptr(), d1["z"], d1["wls"], d1["weights"],
                                     wos.Context(wavelength=d1["wls"][0]), o1.data_ptr())

            def part2(gx=g):
                gx.partially_coherent_dev(n2, d2["dx"], d2["width"], d2["coherence"], m2, nz.data_ptr(), d2["z"],
                                          wos.Context(wavelength=d2["wl"]), o2.data_ptr())

            def part3(gx=g):
                gx.volume_dev(n3, n3, d3["dx"], 1, f3.data_ptr(), d3["zs"], wos.Context(wavelength=d3["wl"]),
                              o3.data_ptr())

            def cfg4_run():
                part1()
                part2()
                part3()
            rec["device_direct_s"] = timed(cfg4_run, max(2, args.steps // 4), 1)
            rec["parts_direct_s"] = {k: timed(f, max(2, args.steps // 4), 1)
                                     for k, f in (("cfg4.1", part1), ("cfg4.2", part2), ("cfg4.3", part3))}
            gr = _graph_of(g, cfg4_run)
            if gr is not None:
                rec["device_sequential_graph_s"] = timed(gr.launch, max(2, args.steps // 4), 1)
                gr.close()
            # the three batches as concurrent branches of one graph: parts 2
            # and 3 on contexts of their own (wos_graph_capture_fork / _join)
            gb, gc = wos.GPU(prec), wos.GPU(prec)
            part2(gb)
            part3(gc)
            gb.synchronize()
            gc.synchronize()
            g.synchronize()
            gr = None
            g.graph_capture_begin()
            try:
                g.graph_capture_fork(gb)
                g.graph_capture_fork(gc)
                part1(g)
                part2(gb)
                part3(gc)
            except Exception:
                pass
            for gx in (gb, gc):
                try:
                    g.graph_capture_join(gx)
                except Exception:
                    pass
            try:
                gr = g.graph_capture_end()
            except Exception:
                gr = None
            if gr is not None:
                rec["device_s"] = timed(gr.launch, max(2, args.steps // 4), 1)
                rec["device_api"] = ("wos_polychromatic_dev, wos_partially_coherent_dev and wos_volume_dev on "
                                     "three contexts, concurrent branches of one graph")
                gr.close()
            else:
                rec["device_s"] = rec.get("device_sequential_graph_s", rec["device_direct_s"])
            gb.close()
            gc.close()
            del nz, o3
            torch.cuda.empty_cache()
            if prec == wos.FP64:
                t0 = time.perf_counter()
                O.polychromatic(O.Field(d1["ex"].copy(), d1["dx"]), d1["z"], d1["wls"][:4], np.ones(4), "asm",
                                O.Context(wavelength=d1["wls"][0]))
                t1 = time.perf_counter()
                modes = O.schell_realizations(n2, d2["dx"], d2["width"], d2["coherence"], d2["noise"][:8])
                for k in range(8):
                    O.propagate(O.Field(modes[k].copy(), d2["dx"]), d2["z"], "asm", O.Context(wavelength=d2["wl"]))
                t2 = time.perf_counter()
                O.propagate3d(O.Field(d3["ex"].copy(), d3["dx"]), d3["zs"][:4], "asm", O.Context(wavelength=d3["wl"]))
                t3 = time.perf_counter()
                # 4 of 64 wavelengths, 8 of 256 modes, 4 of 128 planes, each scaled
                rec_cpu = (t1 - t0) * 16 + (t2 - t1) * m2 / 8 + (t3 - t2) * d3["zs"].size / 4
        elif name == "cfg4.2":
            n, dx, z, m = 512, 4e-6, 0.01, 256
            noise = (rng_noise := np.random.default_rng(1)).standard_normal((m, n, n)) / np.sqrt(2) + \
                1j * rng_noise.standard_normal((m, n, n)) / np.sqrt(2)
            pnoise = torch.from_numpy(noise).pin_memory().numpy()
            pout = torch.zeros((n, n), dtype=torch.float64).pin_memory().numpy()
            rec["e2e_s"] = timed(lambda: g.partially_coherent(n, dx, 600e-6, 50e-6, pnoise, z, "asm",
                                                               wos.Context(wavelength=632.8e-9), out=pout),
                                 max(2, args.steps // 10), 1)
            if prec == wos.FP64:
                t0 = time.perf_counter()
                modes = O.schell_realizations(n, dx, 600e-6, 50e-6, noise[:8])
                for k in range(8):
                    O.propagate(O.Field(modes[k].copy(), dx), z, "asm", O.Context(wavelength=632.8e-9))
                rec_cpu = (time.perf_counter() - t0) * m / 8  # 8 of 256 modes, scaled
        elif name == "cfg4.3":
            n, dx, wl = 768, 4e-6, 632.8e-9
            x = (np.arange(n) - n / 2) * dx
            ex = np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / (300e-6) ** 2).astype(np.complex128)
            zs = np.linspace(0, 0.01, 128)
            hf = wos.Field(torch.from_numpy(ex).pin_memory().numpy(), dx)
            pout = torch.zeros((128, 1, n, n), dtype=torch.complex128).pin_memory().numpy()
            rec["e2e_s"] = timed(lambda: g.volume(hf, zs, "asm", wos.Context(wavelength=wl), out=pout),
                                 max(2, args.steps // 10), 1)
            if prec == wos.FP64:
                t0 = time.perf_counter()
                O.propagate3d(O.Field(ex.copy(), dx), zs[:4], "asm", O.Context(wavelength=wl))
                rec_cpu = (time.perf_counter() - t0) * 32  # 4 of 128 planes, scaled
        elif name == "cfg5":
            n, dx, wl, z = 2048, 4e-6, 633e-9, 0.1
            r = np.random.default_rng(1)
            phi = r.uniform(0, 2 * np.pi, (n, n))
            x = (np.arange(n) - n / 2) * dx
            tgt = np.zeros((n, n))
            for cx, cy in r.uniform(-0.3, 0.3, (16, 2)) * n * dx:
                tgt += np.exp(-((x[None, :] - cx) ** 2 + (x[:, None] - cy) ** 2) / (2 * (20e-6) ** 2))
            a = np.ones((n, n), dtype=np.complex128)
            dt = torch.complex128 if prec == wos.FP64 else torch.complex64
            with torch.cuda.stream(stream):
                ad = torch.from_numpy(a).to(dt).cuda()
                pd = torch.from_numpy(phi).cuda()
                td = torch.from_numpy(tgt).cuda()
                gd = torch.empty((n, n), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            rec["device_s"] = timed(lambda: g.asm_loss_grad_dev(n, n, dx, z, wos.Context(wavelength=wl), ad.data_ptr(),
                                                                pd.data_ptr(), td.data_ptr(), gd.data_ptr()),
                                    args.steps, args.warmup)
            # host entry point on pinned inputs (as a caller with page-locked buffers would pass them)
            pin = lambda x: torch.from_numpy(x).pin_memory().numpy()  # noqa: E731
            ah, ph, th = pin(a), pin(phi), pin(tgt)
            rec["e2e_s"] = timed(lambda: g.asm_loss_grad(ah, ph, th, dx, z, wos.Context(wavelength=wl)),
                                 max(2, args.steps // 10), 1)
            if prec == wos.FP64:
                rec_cpu = cpu(lambda: O.asm_phase_loss_grad(a, phi, tgt, dx, z, O.Context(wavelength=wl)))
        elif name == "train":
            # an element train at 2048^2: lens, 5 cm, aperture, 2 cm, grating, 1 cm, sensor
            n, dx, wl = 2048, 2e-6, 632.8e-9
            r = np.random.default_rng(1)
            pin = lambda x: torch.from_numpy(x).pin_memory().numpy()  # noqa: E731
            ex = pin(np.exp(1j * r.uniform(0, 2 * np.pi, (n, n))))
            sensor = pin(np.zeros((n, n)))
            ops = [("lens", wl, 0.1, 1.5e-3, 0.0, 0.0), ("propagate", 0.05, "asm"), ("aperture", 1.2e-3, 0.0, 0.0, 0.0),
                   ("propagate", 0.02, "asm"), ("grating", "phase_sin", 40e-6, 1.0, 0.5, 0.0, 0.0, 0.0),
                   ("propagate", 0.01, "asm"), ("intensity", sensor)]
            f = wos.Field(ex, dx)
            cx = wos.Context(wavelength=wl, warnings_enabled=False)
            rec["e2e_s"] = timed(lambda: g.train(f, ops, cx), max(2, args.steps // 10), 1)

            def per_call():
                g.apply_lens(f, wl, 0.1, 1.5e-3)
                g.propagate(f, 0.05, "asm", cx)
                g.apply_aperture_circle(f, 1.2e-3)
                g.propagate(f, 0.02, "asm", cx)
                g.apply_grating(f, "phase_sin", 40e-6, 1.0, 0.5)
                g.propagate(f, 0.01, "asm", cx)
            rec["one_call_per_op_s"] = timed(per_call, max(2, args.steps // 10), 1)
            if prec == wos.FP64:
                def cpu_train():
                    of = O.Field(ex.copy(), dx)
                    oc = O.Context(wavelength=wl, warnings_enabled=False)
                    O.apply_lens(of, wl, 0.1, 1.5e-3)
                    O.propagate(of, 0.05, "asm", oc)
                    O.apply_aperture_circle(of, 1.2e-3)
                    O.propagate(of, 0.02, "asm", oc)
                    O.apply_grating(of, "phase_sin", 40e-6, 1.0, 0.5)
                    O.propagate(of, 0.01, "asm", oc)
                    of.intensity()
                rec_cpu = cpu(cpu_train)
        elif name == "cfg5.2":
            # 3 phase masks, each followed by 200 BPM slices of 5 um through a
            # uniform n = 1.5 medium; loss and gradient of all masks
            n, dx, wl, nl, S, dz = 2048, 4e-6, 633e-9, 3, 200, 5e-6
            r = np.random.default_rng(1)
            phis = r.uniform(0, 2 * np.pi, (nl, n, n))
            x = (np.arange(n) - n / 2) * dx
            tgt = np.zeros((n, n))
            for cx, cy in r.uniform(-0.3, 0.3, (16, 2)) * n * dx:
                tgt += np.exp(-((x[None, :] - cx) ** 2 + (x[:, None] - cy) ** 2) / (2 * (20e-6) ** 2))
            a = np.ones((n, n), dtype=np.complex128)
            desc = wos.IndexDesc()
            desc.re_bg = 1.5
            dt = torch.complex128 if prec == wos.FP64 else torch.complex64
            with torch.cuda.stream(stream):
                ad = torch.from_numpy(a).to(dt).cuda()
                pd = torch.from_numpy(phis).cuda()
                td = torch.from_numpy(tgt).cuda()
                gd = torch.empty((nl, n, n), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            cx = wos.Context(wavelength=wl)
            rec["device_s"] = timed(lambda: g.bpm_stack_loss_grad_dev(ad.data_ptr(), pd.data_ptr(), td.data_ptr(),
                                                                      gd.data_ptr(), nl, n, n, dx, S * dz, S, desc,
                                                                      cx),
                                    max(2, args.steps // 10), 1)
            pin = lambda x: torch.from_numpy(x).pin_memory().numpy()  # noqa: E731
            ah, ph, th = pin(a), pin(phis), pin(tgt)
            rec["e2e_s"] = timed(lambda: g.bpm_stack_loss_grad(ah, ph, th, dx, S * dz, S, desc, cx), 2, 1)
            if prec == wos.FP64:
                od = O.IndexDesc()
                od.re_bg = 1.5
                # one mask and one slice forward + adjoint, scaled to nl * S slices
                rec_cpu = nl * S * cpu(lambda: O.bpm_stack_loss_grad(a, phis[:1], tgt, dx, dz, 1, od,
                                                                     O.Context(wavelength=wl)))
        g.close()
        lines.append(rec)

    f32, f64 = lines
    best = f32["device_s"] if "device_s" in f32 else f32["e2e_s"]
    ab = _algorithmic_bytes(name, 8)
    line = {"metric": f"{name} runs/s (FP32 pipeline; FP64 beside it)", "value": 1.0 / best, "unit": "runs/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": best * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": name, "timing": "device-resident" if "device_s" in f32 else "host API (H2D/D2H included)"},
            "roofline": {"bound": "hbm", "achieved": ab / best / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": ab / best / 1e9 / peak, "algorithmic_bytes_per_run": ab,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"},
            "fp32": f32, "fp64": f64,
            "cpu_baseline": {"value": 1.0 / rec_cpu, "unit": "runs/s", "cores": cores, "kind": "port",
                             "sample": "FP64 C oracle, bounded sample scaled to one run"}}
    print(json.dumps(line), flush=True)

def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--batch", type=int, default=BATCH)
    ap.add_argument("--impl", default="ours")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--config", default="headline",
                    help="headline (default) or one of cfg1 cfg2 cfg3 cfg4 cfg4.1 cfg4.2 cfg4.3 cfg5 cfg5.2 train")
    ap.add_argument("--no-autotune", action="store_true",
                    help="use the default (or WOS_ROWE/WOS_COLE/WOS_COLW) launch configuration")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
        return
    if args.config != "headline":
        run_config(args)
        return

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    wos = importlib.import_module("tetsuhiro-wos_b200")

    stream = torch.cuda.Stream()
    g32 = wos.GPU(wos.FP32, device=local)
    g32.set_stream(stream.cuda_stream)
    g64 = wos.GPU(wos.FP64, device=local)
    g64.set_stream(stream.cuda_stream)
    ctx = wos.Context(wavelength=WL, warnings_enabled=False)  # the reference arm's Context
    # launch configuration of the specialised sweeps: timed on this device
    if args.no_autotune:
        tune32 = tune64 = ("default",) * 3
    else:
        tune32 = g32.autotune(N, N)
        tune64 = g64.autotune(N, N)

    ex = input_field()
    # the FP64 oracle on the same input, on rank 0 before any timed region:
    # its CPU rate and the parity reference
    cpu, ref = None, None
    if rank == 0:
        cpu, ref = cpu_baseline(ex, 1 if args.no_cpu else 3)
        if args.no_cpu:
            cpu = None
    with torch.cuda.stream(stream):
        base32 = torch.from_numpy(ex.astype(np.complex64)).cuda()
        bufs = [base32.clone() for _ in range(POOL)]
    torch.cuda.synchronize()

    # ---- correctness of this exact workload against the oracle, through the
    # calls the timed regions make (autotuned sweeps)
    with torch.cuda.stream(stream):
        a32 = base32.clone()
        a64 = torch.from_numpy(ex).cuda()
    torch.cuda.synchronize()
    g32.propagate_batch_dev(N, N, DX, 1, [a32.data_ptr()], [a32.data_ptr()], ZPROP, "asm", ctx)
    g64.propagate_dev(N, N, DX, 1, a64.data_ptr(), a64.data_ptr(), ZPROP, "asm", ctx)
    torch.cuda.synchronize()
    r32 = a32.cpu().numpy().astype(np.complex128)
    r64 = a64.cpu().numpy()
    del a32, a64

    def rel(a, b):
        return float(np.sqrt(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2)))
    parity = {"rel_l2_fp32_vs_fp64_gpu": rel(r32, r64), "tolerance_fp32": 1e-5, "tolerance_fp64": 1e-12,
              "reference": "FP64 C oracle on the same input and Context"}
    if ref is not None:
        parity["rel_l2_fp32_vs_oracle"] = rel(r32, ref)
        parity["rel_l2_fp64_vs_oracle"] = rel(r64, ref)

    # ---- FP64 kernel on the same workload (reported beside the headline)
    with torch.cuda.stream(stream):
        bufs64 = [torch.from_numpy(ex).cuda() for _ in range(8)]
    torch.cuda.synchronize()
    s64 = max(4, args.steps // 2)
    # the same API as the headline (device batch, two streams), and one
    # wos_propagate_dev call per field beside it
    ms64, _ = time_batch(g64, torch, bufs64, s64, 3, 32, ctx, stream)
    fp64_rate = s64 * 32 / (ms64 / 1e3)
    ms64s, _, _ = time_device(g64, torch, bufs64, s64, 2, 32, ctx, stream)
    fp64_single = s64 * 32 / (ms64s / 1e3)
    del bufs64
    torch.cuda.empty_cache()

    # ---- headline: device-resident FP32
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    ms, launches = time_batch(g32, torch, bufs, args.steps, args.warmup, args.batch, ctx, stream)
    clk = clocks.stop()
    # one wos_propagate_dev call per field, in order on one stream
    s1 = max(2, args.steps // 4)
    ms1, _, _ = time_device(g32, torch, bufs, s1, 1, POOL, ctx, stream)
    single_rate = s1 * POOL / (ms1 / 1e3)
    # per-kernel durations from a separate pass with per-launch events (the
    # events would add gaps to the headline region)
    _, _, prof = time_device(g32, torch, bufs, s1, 1, POOL, ctx, stream, profile=True)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    props = args.steps * args.batch * world
    value = props / (ms_max / 1e3)

    # ---- the second input of the workload: the lens recipe (Gaussian clipped
    # by an aperture, thin-lens phase), its parity and the same timed batch
    lens = WL_.lens_beam(N)
    lens_rec = {"input": "Gaussian w = 200 um clipped at r = 400 um, thin lens f = 0.2 m"}
    with torch.cuda.stream(stream):
        l32 = torch.from_numpy(lens.astype(np.complex64)).cuda()
        l64 = torch.from_numpy(lens).cuda()
    torch.cuda.synchronize()
    g32.propagate_batch_dev(N, N, DX, 1, [l32.data_ptr()], [l32.data_ptr()], ZPROP, "asm", ctx)
    g64.propagate_dev(N, N, DX, 1, l64.data_ptr(), l64.data_ptr(), ZPROP, "asm", ctx)
    torch.cuda.synchronize()
    if rank == 0:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O  # noqa: E402  (checker only)
        lo = O.Field(lens.copy(), DX)
        O.propagate(lo, ZPROP, "asm", oracle_context(O))
        lens_rec["rel_l2_fp32_vs_oracle"] = rel(l32.cpu().numpy().astype(np.complex128), lo.ex)
        lens_rec["rel_l2_fp64_vs_oracle"] = rel(l64.cpu().numpy(), lo.ex)
    with torch.cuda.stream(stream):
        lin = torch.from_numpy(lens.astype(np.complex64)).cuda()
        for b in bufs:
            b.copy_(lin)
    torch.cuda.synchronize()
    del l32, l64, lin
    ms_l, _ = time_batch(g32, torch, bufs, args.steps, args.warmup, args.batch, ctx, stream)
    tl = torch.tensor([ms_l], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(tl, op=dist.ReduceOp.MAX)
    lens_rec["value"] = props / (float(tl.item()) / 1e3)
    lens_rec["unit"] = "props/s"

    # roofline of the dominant kernel: algorithmic bytes per launch / mean launch time
    peak, peak_kind = measured_peaks()
    per_launch_bytes = {"row_fwd": 16 * N * N, "col_fused": 16 * N * N, "row_inv": 16 * N * N}
    dom = max(prof, key=lambda k: prof[k][0]) if prof else None
    roof = None
    if dom:
        tot_ms, cnt = prof[dom]
        avg_s = tot_ms / cnt / 1e3
        ach = per_launch_bytes.get(dom, 16 * N * N) / avg_s / 1e9
        roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic": None, "algorithmic_bytes_per_launch": per_launch_bytes.get(dom),
                "mean_launch_us": avg_s * 1e6,
                "per_kernel_us": {k: v[0] / v[1] * 1e3 for k, v in prof.items()},
                "whole_propagation": {"algorithmic_bytes": 48 * N * N,
                                      "achieved_gbs": 48 * N * N * value / world / 1e9,
                                      "frac": 48 * N * N * value / world / 1e9 / peak},
                # secondary byte models: the compulsory I/O of a propagation
                # (read and write the field once) and the classic four sweeps
                "compulsory_io": {"bytes": 16 * N * N, "achieved_gbs": 16 * N * N * value / world / 1e9,
                                  "frac": 16 * N * N * value / world / 1e9 / peak},
                "four_sweeps": {"bytes": 64 * N * N, "achieved_gbs": 64 * N * N * value / world / 1e9,
                                "frac": 64 * N * N * value / world / 1e9 / peak}}
    traffic_file = os.path.join(ROOT, "profiles", "traffic_asm2048_c64.json")
    if roof and os.path.exists(traffic_file):
        try:
            with open(traffic_file) as fh:
                roof["traffic"] = json.load(fh).get(dom)
        except Exception:
            pass

    # ---- end to end through the host API (complex128 host buffers, the
    # same Context): one wos_propagate_batch call over E2E_FIELDS fields per
    # step (uploads, sweeps and downloads of consecutive fields overlap), and
    # one wos_propagate call per field beside it; page-locked host buffers (the
    # contract's e2e) and pageable ones (numpy arrays, as a Go slice is)
    e2e = None
    if not args.no_e2e:
        # 32 fields a call: a call pays the pipeline's fill and drain once
        # (the first upload and the last download run alone, ~1.3 ms), 11 %
        # of a call of 8 fields and 3 % of one of 32
        E2E_FIELDS = 32

        def e2e_time(fn, n):
            fn()
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for _ in range(n):
                fn()
            t1.record(stream)
            torch.cuda.synchronize()
            te = torch.tensor([t0.elapsed_time(t1)], dtype=torch.float64, device="cuda")
            if world > 1:
                dist.all_reduce(te, op=dist.ReduceOp.MAX)
            return float(te.item()) / 1e3

        def e2e_leg(pinned: bool) -> dict:
            fields = []
            for _ in range(E2E_FIELDS):
                h = torch.from_numpy(ex.copy())
                h = h.pin_memory() if pinned else h
                f = wos.Field(ex, DX)
                f.ex = h.numpy()  # the host buffer itself (no copy)
                fields.append(f)
            nb = max(2, args.steps // 4)
            tb = e2e_time(lambda: g32.propagate_batch(fields, ZPROP, "asm", ctx), nb)
            ns = max(3, args.steps // 2)
            ts = e2e_time(lambda: g32.propagate(fields[0], ZPROP, "asm", ctx), ns)
            kind = "page-locked" if pinned else "pageable"
            return {"value": nb * E2E_FIELDS * world / tb, "unit": "props/s",
                    "h2d_bytes_per_step": N * N * 16 * E2E_FIELDS, "d2h_bytes_per_step": N * N * 16 * E2E_FIELDS,
                    "api": f"wos_propagate_batch over {E2E_FIELDS} {kind} host complex128 fields per step",
                    "single_call": {"value": ns * world / ts, "unit": "props/s",
                                    "api": f"one wos_propagate per {kind} host field"}}
        e2e = e2e_leg(True)
        e2e["pageable"] = e2e_leg(False)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "props/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": workload_config(), "fields_per_step": args.batch,
                "autotune": {"fp32": {"row_e": tune32[0], "col_e": tune32[1], "col_w": tune32[2]},
                             "fp64": {"row_e": tune64[0], "col_e": tune64[1], "col_w": tune64[2]}},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches, "clocks": clk,
                "fp64": {"value": fp64_rate, "unit": "props/s", "dtype": "f64",
                         "api": "wos_propagate_batch_dev, as the headline",
                         "fp32_speedup": value / world / fp64_rate,
                         "single_call": {"value": fp64_single, "unit": "props/s",
                                         "api": "one wos_propagate_dev per field, one stream"}},
                "single_call": {"value": single_rate * world, "unit": "props/s",
                                "api": "one wos_propagate_dev per field, one stream"},
                "parity": parity,
                "lens_input": lens_rec}
        print(json.dumps(line), flush=True)
    g32.close()
    g64.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
