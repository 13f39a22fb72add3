#!/usr/bin/env python
"""Throughput of the B200 spectral PFC step (Mcell-steps/s).

Workload: plain conserved PFC at 512^3 on one B200, FP32 bulk arithmetic with
FP64 operator tables / k = 0 mode (dx = pi/4, dt = 0.5, r = -0.25, psi0 =
-0.285 + U(-0.01, 0.01), seed 7: the 512^3 case of the "256^3 and 512^3"
configuration).  A step is one PFC time step over the whole grid with the
state resident in HBM.  Every array (0.54 GB each) is larger than the 126 MB
L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With N > 1 (torchrun, one rank per GPU) every rank evolves its own independent
512^3 field (replicas: a single field's FFT does not shard without an all-to-all,
and the path has none); value = all cells of all ranks * K / max-over-ranks time.

--impl reference times the reference algorithm's CPU implementation on this
host's cores instead: the FP64 C restatement of the reference path (the
reference's own FFTW/HeFFTe/MPI build cannot be built here), same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 512
DX = [math.pi / 4] * 3
DT, R, N0, AMP, SEED = 0.5, -0.25, -0.285, 0.01, 7
METRIC = "Mcell-steps/s at 512^3 FP32 vs FP64 GPU (<=1e-5 rel-L2); FFT-pass HBM % of peak"
WORKLOAD = "plain conserved PFC 512^3, FP32 bulk, dx=pi/4 dt=0.5 r=-0.25"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """SM clocks and throttle reasons sampled during a region: NVML polled every
    few milliseconds from a thread (read-only queries), or nvidia-smi where the
    NVML binding is missing."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, device: int, period_s: float = 0.002):
        self.device = device
        self.period = period_s
        self.p = None
        self.nv = None
        self.samples = []  # (sm_mhz, max_mhz, reasons bitmask)
        self.lines = []

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uid = "GPU-" + str(torch.cuda.get_device_properties(self.device).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def __enter__(self):
        import threading
        self.stop = threading.Event()
        try:
            nv, h = self._nvml_handle()
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)

            def poll():
                while not self.stop.is_set():
                    try:
                        self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), smax, reasons(h)))
                    except Exception:
                        pass
                    time.sleep(self.period)

            self.nv = nv
            self.t = threading.Thread(target=poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nv = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(self.device), "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
            return self

        def reader():
            for line in self.p.stdout:
                if line.strip():
                    self.lines.append(line)

        self.t = threading.Thread(target=reader, daemon=True)
        self.t.start()
        t0 = time.time()
        while not self.lines and time.time() - t0 < 3.0:  # first sample before the region
            time.sleep(0.01)
        self.lines.clear()
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.nv is not None:
            self.t.join(timeout=2)
        if self.p:
            time.sleep(0.15)
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, smax, reasons = [], None, set()
        for mhz, mx, bits in self.samples:
            sm.append(float(mhz))
            smax = float(mx)
            for nm, b in self.BITS.items():
                if int(bits) & b:
                    reasons.add(nm)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.samples else ("nvidia-smi" if self.lines else None)}


# z-update variants (opfc_autotune): 0/2 stream per-mode FP64-built tables,
# 1 radial FP64-built tables (L2), 3-5 compute opL/opN per mode in the compute
# precision, 6-8 read the folded FP64-built tables
def operator_source(var_z):
    if var_z in (3, 4, 5):
        return "opL/opN computed per mode in the compute precision (expm1f, fast divide)"
    if var_z in (6, 7, 8, 9):
        return "FP64-built opL/opN tables rounded to FP32 (folded by the evenness of k^2 in ky, kz)"
    if var_z == 1:
        return "FP64-built opL/opN radial tables rounded to FP32"
    return "FP64-built per-mode opL/opN tables rounded to FP32"


def z_table_bytes(var_z, n, t, st):
    """HBM bytes of operator tables one z update reads: t per-mode tables for
    the table variants (0, 2); the folded tables, (M+1)(N/2+1)^2 modes read once
    per step (tiles walked in (ky, N - ky) pairs), for 6-9; none for the radial
    (L2-resident) and computed variants."""
    if var_z in (0, 2):
        return (n // 2 + 1) * n * n * t * st
    if var_z in (6, 7, 8, 9):
        return (n // 2 + 1) * (n // 2 + 1) * (n // 2 + 1) * t * st
    return 0


def alg_bytes_per_kernel(n, prec_bytes, table_bytes):
    """Algorithmic HBM bytes per launch of each kernel of the plain step: every
    pass reads and writes each complex mode once; the z update also reads and
    writes psi_hat and reads `table_bytes` of operator tables."""
    nc = (n // 2 + 1) * n * n
    sc = 2 * prec_bytes
    return {"y_inverse": 2 * nc * sc, "x_fused": 2 * nc * sc, "y_forward": 2 * nc * sc,
            "z_update": nc * 4 * sc + table_bytes, "hermitian_fix": 4 * 2 * n * n * sc}


def cpu_baseline(psi0, budget_s=30.0):
    """Time the FP64 C restatement of the reference step on all host threads."""
    from oracle import oracle as O
    O.set_threads(len(os.sched_getaffinity(0)))
    threads = O.get_threads()
    psi = np.ascontiguousarray(psi0, dtype=np.float64).copy()
    t1 = O.time_plain(psi, DX, R, DT, 1)
    steps, total = 1, t1
    if t1 * 2 < budget_s:
        k = max(1, min(5, int((budget_s - t1) / max(t1, 1e-9))))
        total = O.time_plain(psi, DX, R, DT, k)
        steps = k
    cells = psi.size
    return {"value": cells * steps / total / 1e6, "unit": "Mcell-steps/s", "cores": threads,
            "kind": "port",
            "sample": f"{steps} plain PFC step(s) at {N}^3 FP64 (C restatement of the reference "
                      f"path, OpenMP {threads} threads), {total:.2f} s"}


def run_reference(args):
    """The reference algorithm's CPU path on this host's cores: the FP64 C
    restatement of the plain PFC step (the reference's own FFTW/HeFFTe/MPI build
    cannot be built here), on the same 512^3 workload and initial condition (the
    oracle's noise generator equals the product's bit for bit).  Nothing of the
    product package is imported in this process.  W untimed warm-up steps, then
    up to K timed steps bounded to ~150 s."""
    ws, rank, _ = dist()
    if rank != 0:
        return 0
    from oracle import oracle as O
    # every host thread this process may run on (torchrun sets OMP_NUM_THREADS=1)
    O.set_threads(len(os.sched_getaffinity(0)))
    psi = O.ic_noise((N, N, N), N0, AMP, SEED)
    threads = O.get_threads()
    t1 = O.time_plain(psi, DX, R, DT, 1)  # first step: paging and thread start-up
    w = max(0, min(args.warmup - 1, int(60.0 / max(t1, 1e-9))))
    if w:
        O.time_plain(psi, DX, R, DT, w)
    k = max(1, min(args.steps, int(150.0 / max(t1, 1e-9))))
    t = O.time_plain(psi, DX, R, DT, k)
    v = psi.size * k / t / 1e6
    line = {"metric": METRIC, "value": v, "unit": "Mcell-steps/s", "n_gpus": 0, "host_threads": threads,
            "steps": k, "warmup": 1 + w, "ms_per_step": 1e3 * t / k, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"plain conserved PFC {N}^3, FP64 CPU, dx=pi/4 dt=0.5 r=-0.25",
                       "n": N, "l2": "arrays larger than L2"},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "Mcell-steps/s", "cores": threads, "kind": "port",
                             "sample": f"{k} plain PFC steps at {N}^3 FP64 after {1 + w} warm-up step(s), "
                                       f"C restatement of the reference path (FFTW/HeFFTe/MPI absent), "
                                       f"{threads} threads"},
            "e2e": {"value": v, "unit": "Mcell-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def timed_steps(model, steps, warmup, ws, stream, repeats=1, reset=None):
    """W warm-up steps, then `repeats` timed regions of exactly `steps` steps,
    each bracketed by a barrier and a device synchronize and timed with CUDA
    events on the handle's stream; returns (median ms, all ms), max over ranks.
    `reset` (untimed, before every region) restores the initial field, for
    workloads whose dynamics must not run longer than one region."""
    import torch
    from openpfc_b200.parallel_plan import max_over_ranks
    if reset:
        reset()
    model.step(warmup)
    model.sync()
    times = []
    for _ in range(repeats):
        if reset:
            reset()
            model.sync()
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        model.step(steps)
        e1.record(stream)
        e1.synchronize()
        model.sync()
        torch.cuda.synchronize()
        times.append(max_over_ranks(e0.elapsed_time(e1), device="cuda"))
    return statistics.median(times), times


def run_b200(args):
    import torch
    import openpfc_b200 as ob
    ws, rank, local = dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local))
    hbm, peak_kind = peaks()
    cells = N ** 3
    psi0 = ob.ic_noise((N, N, N), N0, AMP, SEED + rank)
    psi0_32 = psi0.astype(np.float32)

    m = ob.PfcB200((N, N, N), DX, r=R, precision=ob.FP32, device=local)
    m.initialize(DT)
    # kernel variant per pass, timed on this GPU (untimed set-up); --no-autotune
    # keeps the cached or default choice (OPFC_Y_VARIANT / OPFC_Z_VARIANT force one)
    tune32 = None if args.no_autotune else m.autotune()
    m.set_psi(psi0_32)
    stream = torch.cuda.ExternalStream(m.stream, device=torch.device("cuda", local))
    # clocks are sampled from the warm-up through the end of the timed region
    with Clocks(local) as ck:
        ms, reps_ms = timed_steps(m, args.steps, args.warmup, ws, stream, repeats=args.repeats)
    value = ws * cells * args.steps / (ms / 1e3) / 1e6
    kps = m.kernels_per_step()

    extra = {}
    # FP64 step (same workload) and FP32-vs-FP64 accuracy after 100 steps
    if not args.no_fp64:
        m64 = ob.PfcB200((N, N, N), DX, r=R, precision=ob.FP64, device=local)
        m64.initialize(DT)
        m64.autotune()
        m64.set_psi(psi0_32.astype(np.float64))
        s64 = max(3, min(args.steps, 20))
        ms64, _ = timed_steps(m64, s64, min(args.warmup, 3), ws, torch.cuda.ExternalStream(
            m64.stream, device=torch.device("cuda", local)), repeats=3)
        v64 = ws * cells * s64 / (ms64 / 1e3) / 1e6
        extra["fp64"] = {"value": v64, "ms_per_step": ms64 / s64, "steps": s64}
        extra["fp32_over_fp64"] = value / v64
        if rank == 0:
            acc_steps = 100
            m.set_psi(psi0_32)
            m64.set_psi(psi0_32.astype(np.float64))
            m.step(acc_steps)
            m64.step(acc_steps)
            m.sync()
            m64.sync()
            a = m.get_psi()
            b = m64.get_psi()
            extra["rel_l2_fp32_vs_fp64"] = float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))
            extra["rel_l2_steps"] = acc_steps
            del a, b
        del m64

    # e2e through the public API with host buffers: per step the field goes
    # host -> device (set_psi), one step, device -> host (get_psi), pinned memory
    e2e = None
    if not args.no_e2e:
        host_in = torch.from_numpy(psi0_32.copy()).pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        hin, hout = host_in.numpy(), host_out.numpy()
        k_e2e = max(2, min(args.steps, 5))
        m.set_psi(hin)
        m.step(1)
        m.get_psi(hout)
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(k_e2e):
            m.set_psi(hin)
            m.step(1)
            m.get_psi(hout)
        torch.cuda.synchronize()
        t_e2e = time.perf_counter() - t0
        if ws > 1:
            t = torch.tensor([t_e2e], device="cuda", dtype=torch.float64)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            t_e2e = float(t.item())
        e2e = {"value": ws * cells * k_e2e / t_e2e / 1e6, "unit": "Mcell-steps/s",
               "h2d_bytes_per_step": host_in.numel() * 4, "d2h_bytes_per_step": host_out.numel() * 4,
               "steps": k_e2e, "api": "opfc_set_psi(host) + opfc_step(1) + opfc_get_psi(host)"}

    # per-kernel device time (each kernel alone, CUDA events on the handle's stream)
    m.set_psi(psi0_32)
    prof = m.profile_step(reps=args.profile_reps)
    ab = alg_bytes_per_kernel(N, 4, z_table_bytes(m.variants()[2], N, 2, 4))
    passes = {}
    for k, t in prof.items():
        gbs = ab[k] / (t / 1e3) / 1e9
        passes[k] = {"ms": t, "alg_bytes": ab[k], "gbs": gbs, "frac": gbs / hbm}
    dom = max(prof, key=lambda k: prof[k])
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_512.json")
    if os.path.exists(tpath):
        try:
            # per-launch DRAM bytes from ncu, keyed "<pass>/v<variant>" (the
            # variant of that pass this run uses)
            var = {"y_inverse": m.variants()[0], "y_forward": m.variants()[0], "x_fused": m.variants()[1],
                   "z_update": m.variants()[2]}.get(dom, 0)
            traffic = json.load(open(tpath)).get(f"{dom}/v{var}")
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": passes[dom]["gbs"], "peak": hbm,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": passes[dom]["frac"],
                "traffic": traffic, "alg_bytes": ab[dom]}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(psi0)

    if ws > 1:
        torch.distributed.barrier()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "Mcell-steps/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": WORKLOAD, "operators": operator_source(m.variants()[2]),
                           "n": N, "per_gpu_cells": cells,
                           "l2": "inputs larger than L2 (0.54 GB arrays), no flush",
                           "parallelism": f"replicas x{ws}"},
                "e2e": e2e, "roofline": roofline, "passes": passes, "cpu_baseline": cpu,
                "timing": {"repeats": len(reps_ms), "ms_each": reps_ms, "value_from": "median"},
                "clocks": ck.summary(), "gpu_launches": kps * args.steps,
                "autotune": {"variants_yxz": m.variants(), "ms": tune32}}
        line.update(extra)
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_filtered(args):
    """Mean-field-filtered PFC at 1024^3 FP32: chi = exp(-k^2/(2 0.5^2)),
    N = p2 v^2/2 + p3 v^3/3 + p4 v^4/4 of the filtered density, r = -0.3, seeded
    BCC spheres (8, radius 20 cells) on a liquid n0 = -0.10 + U(-0.001, 0.001)."""
    import torch
    import openpfc_b200 as ob
    n = 1024 if args.n == 512 else args.n
    shape = tuple(args.shape) if args.shape else (n, n, n)
    hbm, peak_kind = peaks()
    t0 = time.time()
    psi0 = ob.ic_seeds(shape, DX, -0.10, 0.001, 8, 20.0, 0.2, 11)
    t_ic = time.time() - t0
    m = ob.FilteredB200(shape, DX, r=-0.3, alpha=0.5, p2=-0.1, p3=-0.5, p4=0.3, precision=ob.FP32)
    m.initialize(DT)
    tune = None if args.no_autotune else m.autotune()
    # The configuration's dynamics are unstable at dt = 0.5 (N grows as psi_MF^4:
    # in the FP64 oracle too, max|psi| doubles about every 5 steps from these
    # seeds and FP32 overflows after ~50 steps), so every timed region restarts
    # from the initial field and runs at most 30 steps; the cost of a step does
    # not depend on the values.
    steps = min(args.steps, 30)
    stream = torch.cuda.ExternalStream(m.stream)
    with Clocks(0) as ck:
        ms, _ = timed_steps(m, steps, args.warmup, 1, stream, repeats=args.repeats, reset=lambda: m.set_psi(psi0))
    args.steps = steps
    cells = shape[0] * shape[1] * shape[2]
    nc = (shape[0] // 2 + 1) * shape[1] * shape[2]
    prof = m.profile_step(reps=max(2, args.profile_reps // 2))
    var_z = m.variants()[2]
    tab = {0: 3 * nc * 4, 2: 3 * nc * 4}.get(var_z, 0)
    if var_z in (6, 7, 8, 9):
        tab = 3 * 4 * (shape[0] // 2 + 1) * (shape[1] // 2 + 1) * (shape[2] // 2 + 1)
    ab = {"y_inverse": 16 * nc, "x_fused": 16 * nc, "y_forward": 16 * nc,
          "z_update": nc * 32 + tab, "hermitian_fix": 4 * 2 * shape[1] * shape[2] * 8}
    passes = {k: {"ms": t, "gbs": ab[k] / (t / 1e3) / 1e9, "frac": ab[k] / (t / 1e3) / 1e9 / hbm}
              for k, t in prof.items()}
    line = {"metric": "Mcell-steps/s, filtered PFC 1024^3 FP32", "value": cells * args.steps / (ms / 1e3) / 1e6,
            "unit": "Mcell-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"mean-field-filtered PFC {'x'.join(map(str, shape))} FP32, 8 seeds",
                       "operators": operator_source(var_z), "ic_seconds": t_ic,
                       "regions": "each timed region restarts from the initial field (unstable dynamics)"},
            "alg_bytes_per_step": sum(ab.values()), "passes": passes, "peak": hbm, "peak_kind": peak_kind,
            "clocks": ck.summary(), "autotune": {"variants_yxz": m.variants(), "ms": tune}}
    print(json.dumps(line), flush=True)
    return 0


def run_ensemble(args):
    """256 independent plain-PFC members, sides from {32,48,64,80,96}, r ~ U(-0.35,-0.10),
    n0 ~ U(-0.35,-0.20), noise U(-0.01,0.01); 50 steps captured in one CUDA graph;
    tile shapes autotuned; per-member rel-L2 of FP32 against the FP64 ensemble.
    Under torchrun the members are split over the ranks by longest-processing-time
    packing on N^3 log N (no data-path collective); the time is the max over ranks
    and `value` counts every rank's cells."""
    import torch
    import openpfc_b200 as ob
    from openpfc_b200.parallel_plan import max_over_ranks, members_for_rank, sum_over_ranks
    ws, rank, local = dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local))
    rng = np.random.default_rng(4)
    count, steps = 256, 50
    members = []
    for i in range(count):
        s = int(rng.choice([32, 48, 64, 80, 96]))
        members.append({"n": (s, s, s), "dx": DX, "r": float(rng.uniform(-0.35, -0.10)),
                        "n0": float(rng.uniform(-0.35, -0.20)), "seed": 500 + i})
    members = members_for_rank(members, rank, ws)
    count = len(members)
    psi0 = [ob.ic_noise(mb["n"], mb["n0"], 0.01, mb["seed"]) for mb in members]
    out = {}
    for prec in (ob.FP32, ob.FP64):
        e = ob.Ensemble(members, precision=prec, device=local)
        e.initialize(DT)
        tune = e.autotune()
        for i, p in enumerate(psi0):
            e.set_psi(i, p)
        stream = torch.cuda.ExternalStream(e.stream)
        e.step(steps)  # builds and runs the 50-step graph once (warm-up)
        e.sync()
        for i, p in enumerate(psi0):
            e.set_psi(i, p)
        e.step(0)  # prepares the work arrays outside the timed region
        e.sync()
        torch.cuda.synchronize()
        # time one launch of the 50-step graph (barrier on both sides, max over ranks)
        if ws > 1:
            torch.distributed.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e.step(steps)
        e1.record(stream)
        e1.synchronize()
        e.sync()
        ms = max_over_ranks(e0.elapsed_time(e1), device="cuda")
        out[prec] = {"ms": ms, "psi": [e.get_psi(i) for i in range(count)], "cells": e.cells,
                     "variants": e.variants(), "tune_ms": tune}
        del e
    cells = int(sum_over_ranks(out[ob.FP32]["cells"], device="cuda"))
    errs = [float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))
            for a, b in zip(out[ob.FP32]["psi"], out[ob.FP64]["psi"])]
    max_err = max_over_ranks(max(errs) if errs else 0.0, device="cuda")
    if ws > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": "Mcell-steps/s, 256-member uneven ensemble FP32 (50 steps, one graph)",
            "value": cells * steps / (out[ob.FP32]["ms"] / 1e3) / 1e6, "unit": "Mcell-steps/s", "n_gpus": ws,
            "scaling": "strong", "parallelism": f"members split over {ws} rank(s) by LPT, no collective",
            "steps": steps, "ms_per_step": out[ob.FP32]["ms"] / steps, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic", "cells": cells,
            "fp64": {"value": cells * steps / (out[ob.FP64]["ms"] / 1e3) / 1e6},
            "max_member_rel_l2_fp32_vs_fp64": max_err, "variants_fp32": out[ob.FP32]["variants"],
            "autotune_ms_fp32": out[ob.FP32]["tune_ms"]}
    print(json.dumps(line), flush=True)
    return 0


def relaunch_under_torchrun(args, argv):
    """`--gpus N` with N > 1 outside torchrun: re-run this script as N ranks
    (one per GPU, or per CPU process with --dry-run) on this node and return
    the launcher's exit status.  Rank 0 prints the JSON line."""
    import socket
    with socket.socket() as so:  # a free rendezvous port on the loopback address
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + list(argv)
    return subprocess.call(cmd)


def run_dry(args):
    """The launcher without the GPU work: every rank joins a gloo process group,
    the ranks agree on the world size and rank 0 prints the line it would print
    (value 0).  Tests the multi-process path on a machine without GPUs."""
    import datetime
    import torch
    import torch.distributed as tdist
    ws, rank, _ = dist()
    if ws > 1:
        tdist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        t = torch.tensor([1.0])
        tdist.all_reduce(t)
        ranks = int(t.item())
        tdist.destroy_process_group()
    else:
        ranks = 1
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": 0.0, "unit": "Mcell-steps/s", "n_gpus": ranks,
                          "dry_run": True, "scaling": "weak",
                          "config": {"workload": WORKLOAD, "parallelism": f"replicas x{ranks}"}}), flush=True)
    return 0


def run_adjoint(args):
    """Adjoint calibration at 128^3 FP32: target from r* = -0.22, n0* = -0.28
    (seed 3, 200 steps); forward with snapshots every 20 steps and the hand-written
    adjoint at r = -0.25, n0 = -0.285 (gradients w.r.t. r, n0 and psi0).  Timed
    on the host clock around the synchronous API calls (forward_checkpointed,
    adjoint), after one untimed run of both."""
    import torch
    import openpfc_b200 as ob
    n = (128, 128, 128)
    steps, K = 200, 20
    mt = ob.PfcB200(n, DX, r=-0.22, precision=ob.FP64)
    mt.initialize(DT)
    mt.set_psi(ob.ic_noise(n, -0.28, 0.01, 3))
    mt.step(steps)
    target = mt.get_psi().astype(np.float32)
    del mt
    m = ob.PfcB200(n, DX, r=-0.25, precision=ob.FP32)
    m.initialize(DT)
    psi0 = ob.ic_noise(n, -0.285, 0.01, 3).astype(np.float32)
    dev_target = torch.tensor(target, device="cuda")
    out = torch.empty_like(dev_target)
    times = []
    for rep in range(1 + args.repeats):
        m.set_psi(psi0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m.forward_checkpointed(steps, K)
        t1 = time.perf_counter()
        m.get_psi(out)
        g, gr, gn = m.adjoint(out - dev_target)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        if rep:
            times.append((t1 - t0, t2 - t1))
    fwd = statistics.median(t[0] for t in times)
    adj = statistics.median(t[1] for t in times)
    cells = n[0] * n[1] * n[2]
    line = {"metric": "adjoint Mcell-steps/s, 128^3 FP32 (200 steps, snapshots every 20)",
            "value": cells * steps / adj / 1e6, "unit": "Mcell-steps/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic", "steps": steps, "checkpoint_every": K,
            "forward_checkpointed_ms": 1e3 * fwd, "adjoint_ms": 1e3 * adj,
            "adjoint_ms_per_step": 1e3 * adj / steps,
            "note": "adjoint time includes re-running every segment's forward steps from its snapshot",
            "grad_r": gr, "grad_n0": gn, "repeats": len(times)}
    print(json.dumps(line), flush=True)
    return 0


def run_axes(args):
    """Plain batched transforms along y and along z on a --n cube (or --shape),
    FP32 (in place along y; z from A into psi_hat): the same TMA-fed column
    kernel on both axes, so the gap between them is the cost of the axis's row
    stride (kz rows are one kz plane apart: 4 MB at 1024^3).  10 launches per
    region after --warmup launches, median of --repeats regions; 16 B of traffic
    per mode."""
    import torch
    import openpfc_b200 as ob
    from openpfc_b200._lib import lib
    shape = tuple(args.shape) if args.shape else (N, N, N)
    m = ob.PfcB200(shape, DX, r=R, precision=ob.FP32)
    m.initialize(DT)
    tune = None if args.no_autotune else m.autotune()
    psi = torch.full((shape[2], shape[1], shape[0]), N0, dtype=torch.float32, device="cuda")
    psi += AMP * torch.rand_like(psi)
    m.set_psi(psi)
    m.sync()
    del psi
    stream = torch.cuda.ExternalStream(m.stream)
    nc = (shape[0] // 2 + 1) * shape[1] * shape[2]
    hbm, kind = peaks()
    out = {}
    for name, p in (("y_forward", 2), ("z_forward", 6)):
        for _ in range(args.warmup):
            _check_rc(lib().opfc_pass(m._h, p, 0.0, 0))
        regions = []
        for _ in range(args.repeats):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(10):
                _check_rc(lib().opfc_pass(m._h, p, 0.0, 0))
            e1.record(stream)
            torch.cuda.synchronize()
            regions.append(e0.elapsed_time(e1) / 10)
        ms = statistics.median(regions)
        gbs = 16 * nc / (ms / 1e3) / 1e9
        out[name] = {"ms": ms, "gbs": gbs, "frac": gbs / hbm}
    line = {"metric": f"plain y and z transforms, {'x'.join(map(str, shape))} FP32 (GB/s on 16 B per mode)",
            "unit": "GB/s",
            "value": out["z_forward"]["gbs"], "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic", "peak": hbm, "peak_kind": kind, "axes": out,
            "kz_row_stride_bytes": (shape[0] // 2) * shape[1] * 8, "variants_yxz": m.variants(),
            "autotune": tune is not None}
    print(json.dumps(line), flush=True)
    return 0


def _check_rc(rc):
    if rc != 0:
        raise RuntimeError(f"opfc_pass returned {rc}")


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--n", type=int, default=512,
                    help="grid side (512 is the measured workload; smaller sides are for profiling)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--repeats", type=int, default=5,
                    help="timed regions of --steps steps each; value is their median")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-reps", type=int, default=10)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the cached (or default) kernel variants instead of timing them first")
    ap.add_argument("--workload", default="plain", choices=["plain", "filtered", "ensemble", "adjoint", "axes"],
                    help="plain: the measured 512^3 line; filtered: mean-field-filtered 1024^3 FP32; "
                         "ensemble: 256 uneven members, 50 steps in one graph; adjoint: 128^3 FP32 "
                         "calibration (200 steps, snapshots every 20); axes: plain y and z transforms "
                         "of an --n cube")
    ap.add_argument("--shape", type=int, nargs=3, default=None, metavar=("N0", "N1", "N2"),
                    help="filtered and axes workloads: a non-cubic grid (filtered: for profiling one pass "
                         "on a small case)")
    ap.add_argument("--dry-run", action="store_true",
                    help="launch the ranks and print the line without GPU work (gloo; for tests)")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    args.repeats = max(1, args.repeats)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch_under_torchrun(args, argv)
    global N, WORKLOAD
    if args.n != N:
        WORKLOAD = WORKLOAD.replace(f"{N}^3", f"{args.n}^3")
        N = args.n
    if args.dry_run:
        return run_dry(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "filtered":
        return run_filtered(args)
    if args.workload == "ensemble":
        return run_ensemble(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "axes":
        return run_axes(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
