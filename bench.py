#!/usr/bin/env python
"""bench.py -- seconds per self-energy (Sigma) evaluation on B200.

Workload: the GPP plain-FP64 benchmark configuration -- 512 bands, nvband 2,
ncouls 32768, nodes_per_group 20 (ngpown 1638), 3 frequencies, seeded inputs
with the benchmark distributions, evaluated by the band-loop kernel (every
(band, G', G, frequency) quotient, as the reference loop nest
GPP/gpp.cpp:343-390).  One step = one Sigma evaluation through the C ABI with
inputs resident in HBM (2.25 GB, larger than the 126 MB L2, so no flush is
needed).

N = 1: the inputs are bgwsigma.inputs.gpp_seeded (PCG64, seed 1234; the
reference build's own output on them is stored in tests/golden/golden.json).
N > 1 (torchrun, one rank per GPU): one Sigma is split over G' columns, as
BerkeleyGW splits ngpown over MPI tasks (GPP/gpp.cpp:144, 162): rank r
generates its contiguous row block of wtilde / I_eps on its GPU
(gpp_philox(rows=...), counter-based, so no rank generates another's rows),
evaluates its partial achtemp, and the partials are all-gathered over NCCL
and summed in rank order; value = max-over-ranks time per Sigma ("scaling":
"strong").  --replicas instead runs one independent Sigma per GPU ("weak").

Extra lines in the JSON: the factored GPP path, the FF sums at 512 bands /
nvband 2 / ncouls 8192 / ngpown 512 / nFreq 15 / nfreqeval 10, the end-to-end
time through host (pinned) buffers, the FP64 roofline of the dominant kernel
against the in-run measured DFMA/DMMA peaks, and the reference's own OpenMP
CPU build timed on this host's cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "berkeleygw-kernels-cpp_b200"))
sys.path.insert(0, str(REPO))

import numpy as np  # noqa: E402

METRIC = "GPP/FF sec per Sigma & % of FP64/TC peak; mixed vs plain FP64 speedup @ rel err"
GPP_DIMS = dict(number_bands=512, nvband=2, ncouls=32768, nodes_per_group=20)
FF_DIMS = dict(number_bands=512, nvband=2, ncouls=8192, ngpown=512, nFreq=15, nfreqeval=10)
WORKLOAD = ("GPP plain FP64 band loop: number_bands 512, nvband 2, ncouls 32768, nodes_per_group 20 "
            "(ngpown 1638), 3 frequencies")


# ----------------------------------------------------------------- helpers --

class ClockSampler:
    """nvidia-smi samples (200 ms) while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        return self.summary()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def rel_err(got, ref) -> float:
    got = np.atleast_1d(np.asarray(got, dtype=np.complex128))
    ref = np.atleast_1d(np.asarray(ref, dtype=np.complex128))
    return float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))


def traffic_from_profiles(kernel: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summaries
    (a line `TRAFFIC <kernel> <bytes_per_launch>` in profiles/*.md)."""
    for p in sorted((REPO / "profiles").glob("*.md")):
        for line in p.read_text().splitlines():
            parts = line.strip().strip("`").split()
            if len(parts) == 3 and parts[0] == "TRAFFIC" and parts[1] == kernel:
                try:
                    return float(parts[2])
                except ValueError:
                    pass
    return None


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ------------------------------------------------------- reference (CPU) --

def cpu_reference_gpp(reps: int, warmup: int) -> dict:
    """Times `reps` whole noflagOCC_solver calls of the reference's OpenMP
    build (or, where it was not built, the oracle port) on the benchmark
    workload, in a process of its own (oracle/cpu_baseline.py: no torch or
    GPU-library threads share the cores).  Returns its JSON record."""
    d = GPP_DIMS
    cmd = [sys.executable, "-m", "oracle.cpu_baseline", "--bands", str(d["number_bands"]), "--nvband",
           str(d["nvband"]), "--ncouls", str(d["ncouls"]), "--npg", str(d["nodes_per_group"]), "--seed", "1234",
           "--reps", str(reps), "--warmup", str(warmup)]
    r = subprocess.run(cmd, cwd=str(REPO), capture_output=True, text=True, check=True)
    return json.loads(r.stdout.strip().splitlines()[-1])


def config_of(world: int) -> dict:
    """The `config` of both arms' lines (identical keys and values)."""
    return {"workload": WORKLOAD, "global_batch": 1,
            "l2": "inputs 2.25 GB resident in HBM (> 126 MB L2); no flush",
            "parallelism": "one Sigma per step" if world == 1 else f"one Sigma per step over {world} ranks"}


def run_reference_arm(args, world, rank):
    if rank != 0:
        return 0
    rec = cpu_reference_gpp(args.steps, args.warmup)
    times = rec["times_s"]
    value = statistics.median(times)
    sample = (f"{len(times)} whole noflagOCC_solver calls (512 bands each, GPP/gpp.cpp:282-289), one per step, "
              f"median {value:.2f} s (min {min(times):.2f}, max {max(times):.2f}); {args.warmup} untimed warm-up "
              f"calls on the first {rec['warmup_bands']} bands")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.mean(times) * 1e3,
            "higher_is_better": False, "scaling": "weak" if world == 1 or args.replicas else "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded PCG64, benchmark distributions)",
            "config": config_of(world),
            "execution": f"OpenMP 3.0 build of the reference on {rec['cores']} host threads (rank 0 only)",
            "cpu_baseline": {"value": value, "unit": "s", "cores": rec["cores"], "kind": rec["kind"],
                             "sample": sample, "times_s": times},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ ours --

def run_ours(args, world, rank, local):
    import torch
    import bgwsigma as bgw
    from bgwsigma import inputs as I

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
        pg = dist

    def barrier():
        if pg is not None:
            pg.barrier()

    def max_over_ranks(x: float) -> float:
        if pg is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    bgw.load()
    dfma_peak, dmma_peak = bgw.measure_fp64_peak(local)

    # --shard at N = 1 runs the same path with one row block (the gather is
    # then the rank's own partial): everything of the N > 1 step but NCCL.
    sharded = (world > 1 or args.shard) and not args.replicas
    if sharded:
        # This rank's G' row block of the one Sigma, generated on its GPU.
        from bgwsigma import shard as SH
        P_all = GPP_DIMS["ncouls"] // GPP_DIMS["nodes_per_group"]
        rows = SH.column_range(P_all, world, rank)
        d = I.gpp_philox(**GPP_DIMS, seed=1234, rows=rows, device=dev)
        g = d.map_arrays(lambda t: t.cpu().numpy())
        args.quick = True
    else:
        g = I.gpp_seeded(**GPP_DIMS, seed=1234 + rank)
        d = bgw.to_device(g, dev)
        if world > 1:
            args.quick = True
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    out = torch.zeros(3, dtype=torch.complex128, device=dev)
    parts = [torch.zeros(3, dtype=torch.complex128, device=dev) for _ in range(world)]
    total = torch.zeros(3, dtype=torch.complex128, device=dev)

    def gather(local_out):
        """Sharded: all-gathers the ranks' partial achtemp (NCCL, after this
        rank's kernels on `stream`) and sums them in rank order."""
        if not sharded or pg is None:
            return local_out
        with torch.cuda.stream(stream):
            pg.all_gather(parts, local_out)
            total.copy_(parts[0])
            for q in parts[1:]:
                total.add_(q)
        return total

    def sigma_step():
        bgw.noflagOCC_solver(d, stream=sh, out=out, algorithm="bandloop", flags=bgw.FLAG_PROFILE)
        return gather(out)

    # Warm-up.
    for _ in range(args.warmup):
        sigma_step()
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    n0 = bgw.launch_count()
    main_ms = []
    e0.record(stream)
    for _ in range(args.steps):
        res_t = sigma_step()
        main_ms.append(bgw.last_profile()["main_kernel_ms"])
    e1.record(stream)
    torch.cuda.synchronize(dev)
    launches = bgw.launch_count() - n0
    clk = clocks.stop()
    barrier()
    torch.cuda.synchronize(dev)
    elapsed_ms = max_over_ranks(e0.elapsed_time(e1))
    prof = bgw.last_profile()
    ms_per_step = elapsed_ms / args.steps
    value = elapsed_ms / 1e3 / (args.steps * (1 if sharded else world))
    result = res_t.cpu().numpy()

    kernel_ms = statistics.mean(main_ms)
    achieved = prof["flops"] / (kernel_ms * 1e-3) / 1e12
    extra = {}
    roofline = {"bound": "fp64", "achieved": achieved, "peak": dfma_peak, "unit": "TFLOP/s",
                "frac": achieved / dfma_peak, "traffic": traffic_from_profiles("gpp_bandloop_kernel"),
                "kernel": prof["main_kernel"], "kernel_ms": kernel_ms,
                "algorithmic_flops_per_launch": prof["flops"], "algorithmic_bytes_per_launch": prof["main_bytes"],
                "peak_source": "in-run DFMA microkernel (bgw_measure_fp64_peak); MEASURED_PEAKS.json has no FP64 "
                               "entry", "peak_dmma": dmma_peak,
                "flop_convention": "21 flops per (band, G', G, frequency) term, 63 per triple (gpp.cpp:374-383)"}

    # End to end: host (pinned) inputs, H2D + kernels + D2H inside the timed region.
    gp = bgw.to_pinned(g)

    def e2e_call(algorithm):
        r = bgw.noflagOCC_solver(gp, stream=sh, algorithm=algorithm)
        if sharded:  # this rank's partial, gathered and summed on the GPUs, read back
            r = gather(torch.as_tensor(r).to(dev)).cpu().numpy()
        return r

    def time_e2e(algorithm):
        e2e_call(algorithm)
        torch.cuda.synchronize(dev)
        barrier()
        h0 = torch.cuda.Event(enable_timing=True)
        h1 = torch.cuda.Event(enable_timing=True)
        n = max(3, min(args.steps, 10))
        h0.record(stream)
        for _ in range(n):
            res = e2e_call(algorithm)
        h1.record(stream)
        torch.cuda.synchronize(dev)
        return max_over_ranks(h0.elapsed_time(h1)) / 1e3 / (n * (1 if sharded else world)), n, res

    e2e_s, e2e_steps, host_res = time_e2e("bandloop")
    # Bytes the call moves host -> device: wtilde and I_eps whole; of aqsmtemp,
    # aqsntemp and vcoul only the ngpown columns the sum reads (gathered on
    # the host inside the call); the index arrays and wx.
    nbp = g.number_bands * g.ngpown
    h2d = (g.wtilde_array.nbytes + g.I_eps_array.nbytes + 2 * 16 * nbp + 8 * g.ngpown + g.inv_igp_index.nbytes
           + g.indinv.nbytes + g.wx_array.nbytes)
    if pg is not None:  # whole job: every rank's copies
        hb = torch.tensor([float(h2d)], dtype=torch.float64, device=dev)
        pg.all_reduce(hb)
        h2d = float(hb.item())
    e2e = {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 48 * world,
           "steps": e2e_steps, "note": "bgw_noflagOCC_solver (band loop) with BGW_MEMORY_HOST on pinned buffers: "
                                       "per step the call reads the host inputs (aqsmtemp / aqsntemp gathered to "
                                       "the ngpown columns used), copies them H2D, runs the kernels and copies "
                                       "achtemp back"}
    if not args.quick:
        # The drop-in's callers hand over pageable (new[]) buffers.
        gp_pinned = gp
        gp = g
        page_s, page_n, _ = time_e2e("bandloop")
        extra["e2e_pageable"] = {"value": page_s, "unit": "s", "h2d_bytes_per_step": int(h2d),
                                 "d2h_bytes_per_step": 48, "steps": page_n,
                                 "note": "band loop, BGW_MEMORY_HOST on pageable numpy buffers"}
        auto_page_s, _, _ = time_e2e("auto")
        extra["e2e_auto_pageable"] = {"value": auto_page_s, "unit": "s", "h2d_bytes_per_step": int(h2d),
                                      "d2h_bytes_per_step": 48,
                                      "note": "default algorithm on pageable numpy buffers: what the reference's "
                                              "own driver gets through the drop-in"}
        gp = gp_pinned
        auto_s, _, auto_res = time_e2e("auto")
        extra["e2e_auto"] = {"value": auto_s, "unit": "s", "h2d_bytes_per_step": int(h2d),
                             "d2h_bytes_per_step": 48,
                             "note": "default algorithm (factored for the band-independent wx), the drop-in's path"}
    del gp

    # Factored GPP path (band-independent wx): HBM-bound stream.
    if not args.quick:
        for _ in range(2):
            bgw.noflagOCC_solver(d, stream=sh, algorithm="factored", flags=bgw.FLAG_PROFILE)
        fms, fdev = [], []
        for _ in range(args.steps):
            fres = bgw.noflagOCC_solver(d, stream=sh, algorithm="factored", flags=bgw.FLAG_PROFILE)
            p = bgw.last_profile()
            fms.append(p["main_kernel_ms"])
            fdev.append(p["device_ms"])
        fk = statistics.mean(fms)
        extra["gpp_factored"] = {
            "s_per_sigma": statistics.mean(fdev) / 1e3, "kernel": p["main_kernel"], "kernel_ms": fk,
            "roofline": {"bound": "hbm", "achieved": p["main_bytes"] / (fk * 1e-3) / 1e9, "unit": "GB/s",
                         "peak": _hbm_peak(), "frac": p["main_bytes"] / (fk * 1e-3) / 1e9 / _hbm_peak(),
                         "algorithmic_bytes_per_launch": p["main_bytes"],
                         "traffic": traffic_from_profiles("gpp_factored_kernel")},
            "rel_err_vs_bandloop": rel_err(fres.cpu().numpy(), result)}
    # Mixed precision band loop (FP32 quotients, compensated FP64 sums).
    if not args.quick:
        for _ in range(2):
            bgw.noflagOCC_solver(d, stream=sh, algorithm="bandloop", precision="mixed", flags=bgw.FLAG_PROFILE)
        mms = []
        for _ in range(max(3, args.steps // 2)):
            mres = bgw.noflagOCC_solver(d, stream=sh, algorithm="bandloop", precision="mixed",
                                        flags=bgw.FLAG_PROFILE)
            mms.append(bgw.last_profile()["main_kernel_ms"])
        mk = statistics.mean(mms)
        extra["gpp_mixed"] = {"kernel": "gpp_bandloop_kernel<mixed>", "kernel_ms": mk,
                              "speedup_vs_fp64_bandloop": kernel_ms / mk,
                              "achieved_TFLOPs": prof["flops"] / (mk * 1e-3) / 1e12,
                              "rel_err_vs_fp64": rel_err(mres.cpu().numpy(), result)}
        # Adjoint (factored, HBM-bound): dSigma/domega and both [1638][32768] gradients.
        gcot = np.array([0.3 - 1.1j, 0.7 + 0.2j, -0.4 + 0.9j])
        for _ in range(2):
            bgw.noflagOCC_solver_backward(d, gcot, stream=sh, flags=bgw.FLAG_PROFILE)
        ams, adev = [], []
        for _ in range(max(3, args.steps // 2)):
            adj = bgw.noflagOCC_solver_backward(d, gcot, stream=sh, flags=bgw.FLAG_PROFILE)
            p = bgw.last_profile()
            ams.append(p["main_kernel_ms"])
            adev.append(p["device_ms"])
        ak = statistics.mean(ams)
        extra["gpp_adjoint"] = {
            "kernel": p["main_kernel"], "kernel_ms": ak, "s_per_call": statistics.mean(adev) / 1e3,
            "roofline": {"bound": "hbm", "achieved": p["main_bytes"] / (ak * 1e-3) / 1e9, "unit": "GB/s",
                         "peak": _hbm_peak(), "frac": p["main_bytes"] / (ak * 1e-3) / 1e9 / _hbm_peak(),
                         "algorithmic_bytes_per_launch": p["main_bytes"]}}
        # Band-loop adjoint: band-dependent wx (wx[n1] = wx + U[-0.25, 0.25]),
        # every band walked per element.
        import dataclasses
        shift = torch.rand(g.number_bands, dtype=torch.float64, device=d.wx_array.device,
                           generator=torch.Generator(device=d.wx_array.device).manual_seed(5)) * 0.5 - 0.25
        db = dataclasses.replace(d, wx_array=(torch.as_tensor(g.wx_array, device=d.wx_array.device)[None, :]
                                              + shift[:, None]).contiguous(), wx_band_stride=3)
        bgw.noflagOCC_solver_backward(db, gcot, stream=sh, flags=bgw.FLAG_PROFILE)
        bms = []
        for _ in range(2):
            bgw.noflagOCC_solver_backward(db, gcot, stream=sh, flags=bgw.FLAG_PROFILE)
            bms.append(bgw.last_profile()["main_kernel_ms"])
        extra["gpp_adjoint"]["bandloop"] = {
            "kernel": bgw.last_profile()["main_kernel"], "kernel_ms": statistics.mean(bms),
            "wx": "band-dependent (stride 3)",
            "fp64_ops_per_term": 18,
            "fp64_pipe_frac": 18 * 3 * g.number_bands * g.ngpown * g.ncouls / (statistics.mean(bms) * 1e-3)
            / (dfma_peak * 1e12 / 2)}
        del db
        if rank == 0 and not args.no_cpu:
            from oracle.oracle import Oracle
            rw, ri, rd = Oracle().gpp_backward(g, gcot)
            extra["gpp_adjoint"]["rel_err_vs_oracle"] = {
                "grad_wtilde": rel_err(adj[0].cpu().numpy(), rw), "grad_I_eps": rel_err(adj[1].cpu().numpy(), ri),
                "dachtemp_domega": rel_err(adj[2].cpu().numpy(), rd)}
            extra["gpp_mixed"]["rel_err_vs_oracle"] = rel_err(mres.cpu().numpy(), Oracle().gpp(g, factored=True))
        del adj
        # Screened exchange of the occupied bands (bgw_gpp_sigma's asxtemp:
        # the occupied-band sum at +wx and -wx), device-resident, factored.
        for _ in range(2):
            bgw.gpp_sigma(d, stream=sh, algorithm="factored", want_ach=False, flags=bgw.FLAG_PROFILE)
        sdev = []
        for _ in range(max(3, args.steps // 2)):
            _, sx = bgw.gpp_sigma(d, stream=sh, algorithm="factored", want_ach=False, flags=bgw.FLAG_PROFILE)
            sdev.append(bgw.last_profile()["device_ms"])
        bdev = []
        for _ in range(max(3, args.steps // 2)):
            bgw.gpp_sigma(d, stream=sh, algorithm="factored", flags=bgw.FLAG_PROFILE)
            p = bgw.last_profile()
            bdev.append((p["device_ms"], p["main_kernel_ms"]))
        extra["gpp_sx"] = {"output": "asxtemp", "nvband": g.nvband, "s_per_call": statistics.mean(sdev) / 1e3,
                           "achtemp_and_asxtemp_s_per_call": statistics.mean(b[0] for b in bdev) / 1e3,
                           "kernel": p["main_kernel"], "kernel_ms": statistics.mean(b[1] for b in bdev),
                           "hbm_frac": p["main_bytes"] / (statistics.mean(b[1] for b in bdev) * 1e-3) / 1e9
                           / _hbm_peak(),
                           "note": "not in the reference (no flagOCC branch): parity unpinned, checked against "
                                   "the oracle's product form"}
        # The same output from the mixed band loop (FP32 quotients).
        _, sxm = bgw.gpp_sigma(d, stream=sh, algorithm="bandloop", precision="mixed", want_ach=False)
        if rank == 0 and not args.no_cpu:
            from oracle.oracle import Oracle
            sx_ref = Oracle().gpp_sx(g, factored=True)
            extra["gpp_sx"]["rel_err_vs_oracle"] = rel_err(sx.cpu().numpy(), sx_ref)
            extra["gpp_sx"]["rel_err_mixed_vs_oracle"] = rel_err(sxm.cpu().numpy(), sx_ref)
    del d
    torch.cuda.empty_cache()

    # Batched uneven GPP: 64 q-point instances in one graph-replayed launch
    # against 64 sequential single-instance calls (same inputs, on the GPU).
    if not args.quick and not args.no_batch:
        extra["gpp_batched"] = bench_batched(bgw, I, dev, sh, stream, dfma_peak, rank)
        torch.cuda.empty_cache()

    # FF sums.
    if not args.quick:
        f = I.ff_seeded(**FF_DIMS, seed=1234 + rank)
        fd = bgw.to_device(f, dev)
        for _ in range(2):
            bgw.ff_sigma(fd, stream=sh, flags=bgw.FLAG_PROFILE)
        kms, dms = [], []
        for _ in range(args.steps):
            ff_out = bgw.ff_sigma(fd, stream=sh, flags=bgw.FLAG_PROFILE)
            p = bgw.last_profile()
            kms.append(p["main_kernel_ms"])
            dms.append(p["device_ms"])
        fk = statistics.mean(kms)
        ach = p["flops"] / (fk * 1e-3) / 1e12
        extra["ff"] = {
            "workload": "FF: number_bands 512, nvband 2, ncouls 8192, ngpown 512, nFreq 15, nfreqeval 10 "
                        "(achsDtemp + asxDtemp + achDtemp_cor in one call)",
            "s_per_sigma": statistics.mean(dms) / 1e3, "kernel": p["main_kernel"], "kernel_ms": fk,
            "roofline": {"bound": "fp64_tensor", "achieved": ach, "unit": "TFLOP/s", "peak": dmma_peak,
                         "frac": ach / dmma_peak, "algorithmic_flops_per_launch": p["flops"],
                         "algorithmic_bytes_per_launch": p["main_bytes"],
                         "achieved_GBps": p["main_bytes"] / (fk * 1e-3) / 1e9,
                         "traffic": traffic_from_profiles("ff_contract_kernel")}}
        # Mixed precision: integer-slice products on the tcgen05 tensor cores.
        for _ in range(2):
            bgw.ff_sigma(fd, stream=sh, precision="mixed", flags=bgw.FLAG_PROFILE)
        mks, mds = [], []
        for _ in range(args.steps):
            mix_out = bgw.ff_sigma(fd, stream=sh, precision="mixed", flags=bgw.FLAG_PROFILE)
            pm = bgw.last_profile()
            mks.append(pm["main_kernel_ms"])
            mds.append(pm["device_ms"])
        mk = statistics.mean(mks)
        extra["ff_mixed"] = {
            "precision": "mixed: 5 balanced int8 digits per operand, levels 2..6 (15 digit pairs), int32 "
                         "accumulation in tensor memory, FP64 recombination; slices cut inside the tcgen05 kernel",
            "s_per_sigma": statistics.mean(mds) / 1e3, "kernel": pm["main_kernel"], "contraction_ms": mk,
            "speedup_vs_fp64": statistics.mean(dms) / statistics.mean(mds),
            "effective_TFLOPs": pm["flops"] / (mk * 1e-3) / 1e12,
            "rel_err_vs_fp64": {k: rel_err(a.cpu().numpy(), b.cpu().numpy())
                                for k, a, b in zip(("achsDtemp", "asxDtemp", "achDtemp_cor"), mix_out, ff_out)}}
        # Through host buffers (the drop-in's case): synchronous calls on the
        # pageable numpy arrays, inputs staged inside the call.
        bgw.ff_sigma(f)
        t0 = time.perf_counter()
        nh = 3
        for _ in range(nh):
            bgw.ff_sigma(f)
        ff_host_s = (time.perf_counter() - t0) / nh
        # The call reads ekq / dFreqGrid on the host and copies the slices the plan uses.
        ff_h2d = (f.aqsmtemp.nbytes + f.aqsntemp.nbytes + f.vcoul.nbytes + f.I_epsR_array.nbytes
                  + f.I_epsA_array.nbytes + f.inv_igp_index.nbytes + f.indinv.nbytes)
        # Option: iw-dependent wx (nfreqeval distinct outputs), FP64 and mixed.
        piw = {}
        for prec in ("fp64", "mixed"):
            fl = bgw.FLAG_PROFILE | bgw.FLAG_FF_WX_PER_IW
            for _ in range(2):
                bgw.ff_sigma(fd, stream=sh, precision=prec, flags=fl)
            ks, ds = [], []
            for _ in range(max(2, args.steps // 4)):
                out = bgw.ff_sigma(fd, stream=sh, precision=prec, flags=fl)
                pp = bgw.last_profile()
                ks.append(pp["main_kernel_ms"])
                ds.append(pp["device_ms"])
            piw[prec] = (statistics.mean(ks), statistics.mean(ds), out, pp)
        kf, df, of_, pf = piw["fp64"]
        km, dm, om, _ = piw["mixed"]
        extra["ff"]["e2e_host_pageable"] = {
            "value": ff_host_s, "unit": "s", "h2d_bytes_per_step_at_most": int(ff_h2d), "d2h_bytes_per_step": 16 * 21,
            "note": "bgw_ff_sigma on pageable numpy buffers (wall time of the synchronous call): staging + kernels + "
                    "outputs; only the frequency slices the plan reads are copied"}
        extra["ff_per_iw"] = {
            "option": "BGW_FLAG_FF_WX_PER_IW: wx = freqevalmin - ekq + iw*freqevalstep, 10 distinct outputs",
            "fp64": {"s_per_sigma": df / 1e3, "contraction_ms": kf,
                     "TFLOPs": pf["flops"] / (kf * 1e-3) / 1e12, "frac_of_dmma_peak": pf["flops"] / (kf * 1e-3) / 1e12
                     / dmma_peak},
            "mixed": {"s_per_sigma": dm / 1e3, "contraction_ms": km, "speedup_vs_fp64": df / dm,
                      "rel_err_vs_fp64": {k: rel_err(a.cpu().numpy(), b.cpu().numpy())
                                          for k, a, b in zip(("achsDtemp", "asxDtemp", "achDtemp_cor"), om, of_)}}}
        if rank == 0 and not args.no_cpu:
            from oracle.oracle import Reference
            if Reference.available():
                ref = Reference()
                t0 = time.perf_counter()
                ra = ref.achs(f)
                t1 = time.perf_counter()
                rs = ref.asx(f)
                t2 = time.perf_counter()
                rc = ref.cor(f)
                t3 = time.perf_counter()
                extra["ff"]["cpu_baseline"] = {
                    "kind": "reference", "cores": ref.num_threads(), "unit": "s",
                    "achsDtemp_s": t1 - t0, "asxDtemp_s": t2 - t1, "achDtemp_cor_s": t3 - t2, "value": t3 - t0,
                    "sample": "full FF workload, one run"}
                extra["ff"]["rel_err_vs_reference"] = {
                    "achsDtemp": rel_err(ff_out[0].cpu().numpy(), ra),
                    "asxDtemp": rel_err(ff_out[1].cpu().numpy(), rs),
                    "achDtemp_cor": rel_err(ff_out[2].cpu().numpy(), rc)}
                extra["ff_mixed"]["rel_err_vs_reference"] = {
                    "achsDtemp": rel_err(mix_out[0].cpu().numpy(), ra),
                    "asxDtemp": rel_err(mix_out[1].cpu().numpy(), rs),
                    "achDtemp_cor": rel_err(mix_out[2].cpu().numpy(), rc)}
        del fd

    # Accuracy against the long-double oracle (exact factored identity).
    cpu_baseline = None
    if rank == 0 and not args.no_cpu:
        from oracle.oracle import Oracle
        # Sharded: the gathered result is the whole problem's sum.
        ref = Oracle().gpp(I.gpp_philox(**GPP_DIMS, seed=1234) if sharded else g, factored=True)
        extra["rel_err_vs_oracle"] = {"bandloop": rel_err(result, ref), "e2e_host_path": rel_err(host_res, ref)}
        # The reference build's own output on these inputs (seed 1234), stored
        # with their fingerprint by tests/golden/make_golden.py --full.
        try:
            full = json.loads((REPO / "tests" / "golden" / "golden.json").read_text())["full"]["gpp_benchmark"]
            if full["fingerprint"] == I.fingerprint(g):
                want = np.array([complex(*z) for z in full["reference"]])
                extra["rel_err_vs_reference"] = {"bandloop": rel_err(result, want),
                                                 "e2e_host_path": rel_err(host_res, want)}
        except (OSError, KeyError, ValueError):
            pass
        if world == 1:
            rec = cpu_reference_gpp(1, 1)
            cpu_baseline = {"value": rec["times_s"][0], "unit": "s", "cores": rec["cores"], "kind": rec["kind"],
                            "sample": "one whole noflagOCC_solver call of the workload (512 bands, "
                                      "GPP/gpp.cpp:282-289) in a process of its own, after one untimed warm-up "
                                      f"call on the first {rec['warmup_bands']} bands"}

    if rank == 0:
        data = ("synthetic (seeded Philox4x64-10 generated on the GPUs, benchmark distributions)" if sharded
                else "synthetic (seeded PCG64, benchmark distributions)")
        line = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False,
                "scaling": "strong" if sharded else "weak", "vs_baseline": None, "dtype": "f64", "data": data,
                "config": config_of(world),
                "execution": (f"G' columns split over {world} GPUs (one NCCL all-gather of the partials per step)"
                              if sharded and world > 1 else
                              "G'-split path with one row block (Philox inputs generated on the GPU; no collective "
                              "at one rank)" if sharded else f"{world} independent Sigma evaluation(s), one per GPU"),
                "roofline": roofline, "cpu_baseline": cpu_baseline, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clk, "extra": extra}
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def make_batch_device(I, dev, n=64, seed=4321):
    """The batched workload generated on the GPU: shapes from
    bgwsigma.inputs.batch_shapes (ncouls uniform in {4096, 4608, ..., 32768},
    number_bands in [128, 512], nodes_per_group 20), values by the library's
    counter-based fill (bgw_fill_uniform) with the benchmark distributions."""
    return I.batch_philox(n, seed, device=dev)


def bench_batched(bgw, I, dev, sh, stream, dfma_peak, rank):
    import torch
    insts = make_batch_device(I, dev)
    nbytes = sum(g.nbytes() for g in insts)
    flops = sum(63.0 * g.number_bands * g.ngpown * g.ncouls for g in insts)
    stream_bytes = sum(32.0 * g.ngpown * g.ncouls for g in insts)
    res = {"workload": "64 instances, ncouls uniform in {4096..32768 step 512}, number_bands in [128, 512], "
                       "nodes_per_group 20; inputs generated on the GPU by bgw_fill_uniform (Philox4x64-10)",
           "device_bytes": nbytes}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        for _ in range(reps):
            fn()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        return ev0.elapsed_time(ev1) / 1e3 / reps

    fp64_band_out = None
    for key, alg, prec in (("bandloop", "bandloop", "fp64"), ("factored", "factored", "fp64"),
                           ("bandloop_mixed", "bandloop", "mixed")):
        t0 = time.perf_counter()
        b = bgw.GppBatch(insts, algorithm=alg, precision=prec, stream=sh)
        create_s = time.perf_counter() - t0
        t_batch = timed(lambda: b.execute(stream=sh), 3)
        batch_out = b.execute(stream=sh).cpu().numpy().copy()
        seq_out = np.zeros_like(batch_out)

        def seq():
            for k, g in enumerate(insts):
                r = bgw.noflagOCC_solver(g, algorithm=alg, precision=prec, stream=sh)
                seq_out[k] = r.cpu().numpy()
        t_seq = timed(seq, 1)
        err = max(rel_err(batch_out[k], seq_out[k]) for k in range(len(insts)))
        entry = {"batched_s": t_batch, "sequential_s": t_seq, "speedup_vs_sequential": t_seq / t_batch,
                 "instances_per_s": len(insts) / t_batch, "tuned": b.info(), "create_s": create_s,
                 "max_rel_diff_vs_sequential": err}
        if key == "bandloop":
            fp64_band_out = batch_out
            entry["roofline"] = {"bound": "fp64", "achieved": flops / t_batch / 1e12, "unit": "TFLOP/s",
                                 "peak": dfma_peak, "frac": flops / t_batch / 1e12 / dfma_peak}
        elif key == "factored":
            entry["roofline"] = {"bound": "hbm", "achieved": stream_bytes / t_batch / 1e9, "unit": "GB/s",
                                 "peak": _hbm_peak(), "frac": stream_bytes / t_batch / 1e9 / _hbm_peak()}
        else:
            entry["speedup_vs_fp64_batched"] = res["bandloop"]["batched_s"] / t_batch
            entry["max_rel_err_vs_fp64"] = max(rel_err(batch_out[k], fp64_band_out[k]) for k in range(len(insts)))
        res[key] = entry
        b.close()
    del insts
    return res


def run_only(args, local):
    """Diagnostic mode for profilers: runs one kernel path W + K times on the
    benchmark shapes (GPP bands optionally reduced with --bands) and prints a
    JSON line with the library's per-call timings.  Not the benchmark line."""
    import torch
    import bgwsigma as bgw
    from bgwsigma import inputs as I
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    bgw.load()
    if args.only.startswith("gpp"):
        dims = dict(GPP_DIMS)
        if args.bands:
            dims["number_bands"] = args.bands
        per_band = args.only == "gpp_adjoint_bandloop"
        d = bgw.to_device(I.gpp_seeded(**dims, seed=1234, wx_per_band=per_band), dev)
        if args.only in ("gpp_adjoint", "gpp_adjoint_bandloop"):
            call = lambda: bgw.noflagOCC_solver_backward(d, [1, 1j, -1], flags=bgw.FLAG_PROFILE)  # noqa: E731
        elif args.only == "gpp_sigma":
            call = lambda: bgw.gpp_sigma(d, algorithm="factored", flags=bgw.FLAG_PROFILE)  # noqa: E731
        else:
            alg = "bandloop" if args.only == "gpp_mixed" else args.only.split("_")[1]
            prec = "mixed" if args.only == "gpp_mixed" else "fp64"
            call = lambda: bgw.noflagOCC_solver(d, algorithm=alg, precision=prec,  # noqa: E731
                                                flags=bgw.FLAG_PROFILE)
    else:
        dims = dict(FF_DIMS)
        if args.bands:
            dims["number_bands"] = args.bands
        if args.freqs:
            dims["nFreq"] = args.freqs
        d = bgw.to_device(I.ff_seeded(**dims, seed=1234), dev)
        prec = "mixed" if "mixed" in args.only else "fp64"
        fl = bgw.FLAG_PROFILE | (bgw.FLAG_FF_SLICE_ALL if args.only == "ff_mixed_all" else 0)
        fl |= bgw.FLAG_FF_STAGED if args.only == "ff_mixed_staged" else 0
        fl |= bgw.FLAG_FF_WX_PER_IW if args.only.startswith("ff_per_iw") else 0
        call = lambda: bgw.ff_sigma(d, precision=prec, flags=fl)  # noqa: E731
    for _ in range(args.warmup):
        call()
    profs = []
    for _ in range(args.steps):
        call()
        profs.append(bgw.last_profile())
    ms = statistics.mean(p["main_kernel_ms"] for p in profs)
    print(json.dumps({"only": args.only, "dims": dims, "kernel": profs[-1]["main_kernel"], "kernel_ms": ms,
                      "device_ms": statistics.mean(p["device_ms"] for p in profs), "flops": profs[-1]["flops"],
                      "tflops": profs[-1]["flops"] / (ms * 1e-3) / 1e12, "main_bytes": profs[-1]["main_bytes"],
                      "GBps": profs[-1]["main_bytes"] / (ms * 1e-3) / 1e9}), flush=True)
    return 0


def _hbm_peak() -> float:
    p = REPO / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        return 6650.0  # fallback measurement of this pool


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--quick", action="store_true", help="GPP band loop + e2e only")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline and oracle check")
    ap.add_argument("--replicas", action="store_true",
                    help="with N > 1: one independent Sigma per GPU instead of one Sigma split over G'")
    ap.add_argument("--shard", action="store_true",
                    help="run the G'-split path (per-rank Philox inputs, gather) also at N = 1")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-instances extra")
    ap.add_argument("--only", choices=["gpp_bandloop", "gpp_mixed", "gpp_factored", "gpp_adjoint",
                                       "gpp_adjoint_bandloop", "gpp_sigma", "ff", "ff_mixed",
                                       "ff_mixed_all", "ff_mixed_staged", "ff_per_iw", "ff_per_iw_mixed"],
                    default=None,
                    help="diagnostic: time one kernel path only (for profilers)")
    ap.add_argument("--bands", type=int, default=0, help="with --only: number_bands override")
    ap.add_argument("--freqs", type=int, default=0, help="with --only ff*: nFreq override")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_setup(args)
    if args.only:
        return run_only(args, local)
    if args.impl == "reference":
        return run_reference_arm(args, world, rank)
    return run_ours(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
