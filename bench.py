#!/usr/bin/env python3
"""Benchmark of the WENO path on B200.

Workload (one "step"): FP64 WENO5-JS reconstruction with the MP limiter fused,
x, y and z sweeps, on a 200^3-cell block (m=n=p=199) with v_size=8 and
buff_size=6 -- 3 x 148,135,424 = 444.4 M face states per step.  Inputs are
the seeded smooth-plus-jump field and the true uniform-grid WENO5-JS
coefficients.  Metric: face-states/s (whole job).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the CPU restatement of the reference harness (the
oracle; the Fortran reference cannot be built here) on the host cores.
Multi-GPU (torchrun): every rank owns its own 200^3 x 8 block (weak
scaling); there is no data-path collective.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

M = 199
NV = 8
BUFF = 6
ORDER = 5
METRIC = "WENO5 face-states/s at 199^3 x 8 vars (FP64 WENO5-JS + MP, x/y/z sweeps)"


SCHEME = "js"


def face_states_per_dir(m=None, nv=NV, buff=BUFF, order=None):
    """Face states one sweep writes: vL and vR on the NC core faces (WENO3:
    on every face of the sweep, the reference's is1 range)."""
    m = M if m is None else m
    order = ORDER if order is None else order
    N = m + 2 * buff + 1
    return 2 * (N if order == 3 else N - 6) * N * N * nv


def alg_bytes_per_sweep(m=None, nv=NV, buff=BUFF, elem=8, order=None):
    """Algorithmic HBM bytes of one fused sweep: read the (NC+2H)-long
    stencil window of every column once, write vL and vR on the NC core faces
    (WENO3: the N+2 cells of its 3-point stencils, vL and vR on all N faces)."""
    m = M if m is None else m
    order = ORDER if order is None else order
    N = m + 2 * buff + 1
    if order == 3:
        return (N + 2) * N * N * nv * elem + 2 * N * N * N * nv * elem
    NC = N - 6
    H = max((order - 1) // 2, 2)
    return (NC + 2 * H) * N * N * nv * elem + 2 * NC * N * N * nv * elem


def family():
    return f"WENO{ORDER}-{'TENO' if SCHEME == 'teno' else 'JS'}"


def main_metric(fp32_main):
    """The headline metric (WENO5-JS, FP64); other families and FP32-bulk name themselves."""
    m = METRIC
    if ORDER != 5 or SCHEME != "js":
        m = m.replace("WENO5 face-states", f"WENO{ORDER} face-states").replace("WENO5-JS", family())
    return m.replace("FP64", "FP32-bulk") if fp32_main else m


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """NVML samples of SM clock and throttle reasons during the timed region."""

    REASONS = {
        "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
        "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80,
    }

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.ok = False

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for name, bit in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.005)

    def __enter__(self):
        if self.ok:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                    "samples": len(self.samples)}
        return {"sm_mhz": float(statistics.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0, None
    import datetime

    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    return rank, ws, local, dist


def cpu_info():
    """Host CPU model, logical CPUs available to this process and the OpenMP
    binding in force (stated beside every CPU number)."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        avail = len(os.sched_getaffinity(0))
    except AttributeError:
        avail = os.cpu_count() or 1
    return {"model": model, "nproc": avail, "OMP_PROC_BIND": os.environ.get("OMP_PROC_BIND", ""),
            "OMP_PLACES": os.environ.get("OMP_PLACES", "")}


def cpu_reference_run(steps, warmup, sample_nv=NV, quiet=False):
    """Time the oracle (CPU restatement of the reference path, built -O3 like
    the reference's CPU recipe, f90:33-36) on all host threads: x/y/z
    WENO5-JS + MP from the reshaped fields of `sample_nv` of the 8 variables
    (all 8 by default: the bench's own workload), `warmup` untimed and
    `steps` timed steps (the reference's protocol is warmup 5, bench >= 10)."""
    # thread binding for the oracle's OpenMP runtime (read when it starts)
    os.environ.setdefault("OMP_PROC_BIND", "spread")
    os.environ.setdefault("OMP_PLACES", "threads")
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from wenostandalone_b200 import fields
    oracle.build()
    info = cpu_info()
    threads = info["nproc"]
    oracle.set_threads(threads)
    vf = fields.smooth_jump_field(M, M, M, sample_nv, BUFF, seed=0)
    ins = []
    for d in range(3):
        rs = oracle.reshape(vf, M, M, M, BUFF, d)
        coefs = fields.uniform_weno_coefficients(5, rs.shape[0] - 12)
        L, R = oracle.order1_copy(vf, M, M, M, BUFF, d)
        ins.append((rs, coefs, L, R))
    del vf

    def step():
        for rs, coefs, L, R in ins:
            oracle.reconstruct(rs, coefs, 5, vL=L, vR=R)
            oracle.preserve_monotonicity(rs, L, R)

    for _ in range(warmup):
        step()
    times = []
    for _ in range(max(steps, 1)):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    dt = sum(times) / len(times)
    fs = 3 * face_states_per_dir(nv=sample_nv)
    return {"value": fs / dt, "sec_per_step": dt, "median_sec_per_step": statistics.median(times),
            "cores": threads, "face_states": fs, "cpu": info, "warmup": warmup, "steps": max(steps, 1),
            "sample": f"x/y/z WENO5-JS + MP on 200^3 cells x {sample_nv} of {NV} variables "
                      f"({fs/1e6:.1f} M face states per step) from pre-reshaped fields, warmup {warmup}, "
                      f"{max(steps, 1)} timed steps, {threads} OpenMP threads on {info['model']} "
                      f"(OMP_PROC_BIND={info['OMP_PROC_BIND']}, OMP_PLACES={info['OMP_PLACES']}); "
                      f"oracle built -O3 -ffp-contract=off"}


def run_reference(args):
    rank, ws, _, dist = dist_init()
    if rank != 0:
        return 0
    r = cpu_reference_run(max(args.steps, 10), max(args.warmup, 5))
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": "face-states/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["sec_per_step"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "steps_run": r["steps"], "warmup_run": r["warmup"], "cpu": r["cpu"],
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "WENO5-JS + MP, x/y/z sweeps, 200^3 cells, FP64", "m=n=p": M,
                   "v_size": NV, "buff_size": BUFF},
        "cpu_baseline": {"value": r["value"], "unit": "face-states/s", "cores": r["cores"], "kind": "port",
                         "sample": r["sample"]},
        "e2e": {"value": r["value"], "unit": "face-states/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import _lib as L
    from wenostandalone_b200 import api, fields

    rank, ws, local, dist = dist_init()
    if dist is not None:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local if dist is not None else 0)
    torch.cuda.set_device(dev)
    wsb.lib()

    g = wsb.Grid(M, M, M, NV, BUFF, scheme=wsb.TENO if SCHEME == "teno" else wsb.JS)
    vf_host = fields.smooth_jump_field(M, M, M, NV, BUFF, seed=rank)
    v = torch.from_numpy(vf_host.ravel(order="F")).to(dev)
    coefs = [tuple(torch.from_numpy(c.ravel(order="F")).to(dev)
                   for c in fields.uniform_weno_coefficients(ORDER, g.nc(d))) for d in range(3)]
    # per-face coefficient arrays (weno_sb_weno_dev): those of a grid
    # stretched along every axis (tanh refinement, cells up to 4x narrower,
    # weno_sb_coefficients), or with --coefficients arrays the uniform-grid
    # values repeated on every face
    if args.coefficients == "arrays":
        pf_coefs = coefs
    else:
        pf_coefs = [tuple(torch.from_numpy(np.asarray(c).ravel(order="F")).to(dev) for c in
                          api.weno_coefficients(ORDER, api.stretched_boundaries(M + 1, BUFF, ratio=4.0,
                                                                               centre=0.3 + 0.2 * d)))
                    for d in range(3)]
    cstructs = [api.coefs_struct(c) for c in pf_coefs]
    # the coefficients are face-independent (uniform grid): the sweeps take
    # them from the kernel-parameter bank through weno_sb_weno_uniform_dev
    faces = [api.face_coefs(fields.uniform_weno_coefficients(ORDER, g.nc(d))) for d in range(3)]
    nface = int(np.prod(g.face_shape(0)))
    outs = [(torch.empty(nface, dtype=torch.float64, device=dev),
             torch.empty(nface, dtype=torch.float64, device=dev)) for _ in range(3)]
    stream = torch.cuda.Stream(device=dev)
    sp = int(stream.cuda_stream)
    flags = wsb.F_MP | wsb.F_FOLDED
    fp32_main = args.precision == "fp32"
    pf_main = args.coefficients in ("arrays", "stretched") and not fp32_main
    if fp32_main:
        # FP32-bulk as the timed step: FP32 v_rs_ws per direction (reshaped
        # once, before timing) and FP32 face states
        rs32 = [torch.empty(int(np.prod(g.rs_shape(d))), dtype=torch.float32, device=dev) for d in range(3)]
        for d in range(3):
            api.reshape(g, d, v, rs32[d], stream=sp)
        o32 = [(torch.empty(nface, dtype=torch.float32, device=dev),
                torch.empty(nface, dtype=torch.float32, device=dev)) for _ in range(3)]

    def step(evs=None, per_face=False):
        for d in range(3):
            if evs is not None:
                evs[d][0].record(stream)
            if fp32_main:
                api.weno_uniform(g, d, ORDER, rs32[d], faces[d], o32[d][0], o32[d][1], flags=wsb.F_MP, stream=sp)
            elif per_face or pf_main:
                api.weno(g, d, ORDER, v, cstructs[d], outs[d][0], outs[d][1], flags=flags, stream=sp)
            else:
                api.weno_uniform(g, d, ORDER, v, faces[d], outs[d][0], outs[d][1], flags=flags, stream=sp)
            if evs is not None:
                evs[d][1].record(stream)

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()

    K = args.steps
    per_kernel = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(3)] for _ in range(K)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev.index if dev.index is not None else 0) as clk:
        t_start.record(stream)
        for k in range(K):
            step(per_kernel[k])
        t_end.record(stream)
        torch.cuda.synchronize()
    barrier()
    elapsed_ms = t_start.elapsed_time(t_end)
    if dist is not None:
        t = torch.tensor([elapsed_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    ms_per_step = elapsed_ms / K
    fs_step = 3 * face_states_per_dir()
    value = ws * fs_step / (ms_per_step * 1e-3)

    # dominant kernel: the sweep with the largest summed time
    sums = [sum(per_kernel[k][d][0].elapsed_time(per_kernel[k][d][1]) for k in range(K)) for d in range(3)]
    dk = int(np.argmax(sums))
    dk_ms = sums[dk] / K
    peak, peak_kind = load_peaks()
    ab = alg_bytes_per_sweep(elem=4 if fp32_main else 8)
    achieved = ab / (dk_ms * 1e-3) / 1e9

    # the same step with per-face coefficient arrays (stretched-grid form)
    per_face = None
    if not args.no_extras and not fp32_main and not pf_main:
        for _ in range(3):
            step(per_face=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(K):
            step(per_face=True)
        e1.record(stream)
        torch.cuda.synchronize()
        pf_ms = e0.elapsed_time(e1) / K
        per_face = {"ms_per_step": pf_ms, "value": 3 * face_states_per_dir() / (pf_ms * 1e-3),
                    "entry": "weno_sb_weno_dev (coefficient arrays read per face)",
                    "coefficients": "WENO5-JS of a tanh-stretched grid on every axis (weno_sb_coefficients, "
                                    "cells up to 4x narrower)"}

    # FP32-bulk variant (same sweeps, FP32 v_rs_ws field and face states)
    fp32 = None
    if not args.no_extras and not fp32_main:
        fp32 = measure_fp32_bulk(g, v, faces, outs, stream, K, dev)
        drop = measure_drop_in(g, v, faces, outs, stream, K, dev)
    else:
        drop = None

    # end-to-end through the handle API with pinned host buffers
    e2e = e2e_full = None
    if not (args.no_extras or fp32_main):
        e2e = measure_e2e(g, vf_host, coefs, max(2, min(K, 5)), dev)
        e2e_full = measure_e2e(g, vf_host, coefs, max(2, min(K, 5)), dev, full_download=True)

    # the other workloads of the path (adjoint, batched blocks, mixed precision):
    # single-GPU measurements, taken in one-GPU runs only (with several ranks
    # the others would wait for rank 0 at the closing barrier)
    adjoint = batched = mixed = families = None
    if not args.no_extras and rank == 0 and ws == 1 and not fp32_main:
        Kx = max(3, min(K, 10))
        torch.cuda.empty_cache()
        adjoint = measure_adjoint(dev, Kx)
        torch.cuda.empty_cache()
        batched = measure_batched(dev, Kx)
        torch.cuda.empty_cache()
        mixed = measure_mixed_precision(dev, Kx)
        torch.cuda.empty_cache()
        families = measure_families(g, v, stream, Kx, dev)
        torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu and not fp32_main:
        cpu = cpu_reference_run(steps=10, warmup=5)

    if rank == 0:
        line = {
            "metric": main_metric(fp32_main), "value": value, "unit": "face-states/s", "n_gpus": ws, "steps": K,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32-bulk" if fp32_main else "f64",
            "data": "synthetic",
            "config": {"workload": (f"FP32-bulk {family()} + MP (FP64 beta and weights), x/y/z sweeps of FP32 "
                                    "v_rs_ws" if fp32_main else
                                    f"FP64 {family()} + MP fused, x/y/z sweeps reading v_vf directly "
                                    "(reshape folded)") + f", {M + 1}^3 cells x 8 vars, buff_size 6",
                       "m=n=p": M, "v_size": NV, "buff_size": BUFF,
                       "coefficients": ("uniform-grid WENO5-JS values as per-face device arrays (weno_sb_weno_dev)"
                                        if args.coefficients == "arrays" else
                                        "WENO5-JS of a tanh-stretched grid as per-face device arrays "
                                        "(weno_sb_coefficients, weno_sb_weno_dev)" if pf_main else
                                        "uniform-grid WENO5-JS"),
                       "field": "seeded smooth-plus-jump", "l2": "inputs (663 MB) and outputs (3.7 GB) exceed "
                                                                  "the 126 MB L2; no flush",
                       "parallelism": f"{ws} independent blocks (weak scaling, no collective)"},
            "roofline": {"bound": "hbm", "kernel": (f"sweep_march_tma_kernel<MP,row tiles,float,cp.async loader> "
                                                    f"{'xyz'[dk]} sweep" if fp32_main else
                                                    f"sweep_march_tma_kernel<MP,{'row' if dk == 0 else 'column'} "
                                                    f"tiles,double,TMA loader{',per-face table' if pf_main else ''}> "
                                                    f"{'xyz'[dk]} sweep"),
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6650 GB/s",
                         "alg_bytes_per_launch": ab, "launch_ms": dk_ms,
                         "traffic": None if (fp32_main or pf_main or M != 199 or ORDER != 5 or SCHEME != "js") else read_traffic()},
            "per_sweep_ms": [s / K for s in sums],
            "fp64_issue": (fp64_issue_bound(dk_ms, clk.summary().get("sm_mhz"))
                           if not (fp32_main or pf_main or M != 199 or ORDER != 5 or SCHEME != "js") else None),
            # the per-face form launches the table build and the sweep
            "gpu_launches": (6 if pf_main else 3) * K,
            "clocks": clk.summary(),
        }
        if per_face:
            line["per_face_coefficients"] = per_face
        if fp32:
            line["fp32_bulk"] = fp32
        if drop:
            line["drop_in"] = drop
        if e2e:
            line["e2e"] = e2e
        if e2e_full:
            line["e2e_full_face_states"] = e2e_full
        if adjoint:
            line["adjoint"] = adjoint
        if batched:
            line["batched"] = batched
        if mixed:
            line["mixed_precision"] = mixed
        if families:
            line["families_200cubed"] = families
        if cpu:
            line["cpu_baseline"] = {"value": cpu["value"], "unit": "face-states/s", "cores": cpu["cores"],
                                    "kind": "port", "sample": cpu["sample"], "cpu": cpu["cpu"]}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# Multi-GPU decompositions other than one block per rank (--decomp)
# ---------------------------------------------------------------------------
def zslab_local_field(slab, v_global):
    """The slab's planes of the block's v_vf (a flat tensor in the Fortran
    order (E1, E2, E3, V)): (E1, E2, nz + 2G, V), flat."""
    E3 = v_global.numel() // (slab.E1 * slab.E2 * slab.nv)
    z0, z1 = slab.global_planes()
    return v_global.view(slab.nv, E3, slab.E1 * slab.E2)[:, z0:z1, :].contiguous().view(-1)


def zslab_step(slab, v_local, sweep, group=None):
    """One step of the z-slab decomposition: the ghost-plane exchange with
    the neighbouring slabs, then the slab's x, y and z sweeps (sweep(d))."""
    slab.exchange(v_local, group)
    for d in range(3):
        sweep(d)


def batch_assignment(blocks, world):
    """The batched workload's blocks per rank, longest-processing-time first
    on their face states (every block's x, y and z sweeps stay on one rank)."""
    from wenostandalone_b200 import sharding
    costs = []
    for cells, nv, order, _scheme in blocks:
        N = [c + 2 * BUFF for c in cells]
        fs = 0
        for d in range(3):
            ns = N[d]
            nf = ns if order == 3 else ns - 6
            fs += 2 * nf * (N[0] * N[1] * N[2] // ns) * nv
        costs.append(fs * (1.5 if order == 7 else 1.0))
    return sharding.lpt_assign(costs, world)


def run_decomp(args):
    """--decomp zslab: one 200^3 x 8 block split along z over the ranks
    (strong scaling): per step every rank exchanges G = buff_size + 3 ghost
    planes with its neighbours (NCCL point-to-point over NVLink; torch's
    P2P calls on the sweeps' stream) and sweeps its slab in x, y and z
    (FP64 WENO5-JS + MP, folded).  --decomp batch: the 96-block batched
    workload placed on the ranks by LPT, one graph launch per rank per step
    (strong scaling).  value = the face states of the whole job / the
    slowest rank's device time per step."""
    import datetime

    import torch

    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import api, fields, sharding
    rank, ws, local, dist = dist_init()
    if dist is not None:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local if dist is not None else 0)
    torch.cuda.set_device(dev)
    wsb.lib()
    stream = torch.cuda.Stream(device=dev)
    sp = int(stream.cuda_stream)
    K = args.steps
    if args.decomp == "zslab":
        slab = sharding.ZSlab(M, M, M, NV, BUFF, ws, rank)
        v_global = fields.smooth_jump_field_dev(M, M, M, NV, BUFF, seed=0, device=dev)
        v = zslab_local_field(slab, v_global)
        del v_global
        g = wsb.Grid(M, M, slab.p_local, NV, BUFF)
        faces = [api.face_coefs(fields.uniform_weno_coefficients(5, g.nc(d))) for d in range(3)]
        outs = [tuple(torch.empty(int(np.prod(g.face_shape(d))), dtype=torch.float64, device=dev)
                      for _ in range(2)) for d in range(3)]

        def sweep(d):
            api.weno_uniform(g, d, 5, v, faces[d], outs[d][0], outs[d][1], flags=wsb.F_MP | wsb.F_FOLDED,
                             stream=sp)

        def step():
            with torch.cuda.stream(stream):
                zslab_step(slab, v, sweep)
        fs_total = 3 * face_states_per_dir()
        launches = 3
        workload = (f"FP64 WENO5-JS + MP, one {M + 1}^3 x {NV} block split along z over {ws} ranks "
                    f"({slab.nz}-cell slabs + {slab.G} ghost planes a side, exchanged each step by NCCL P2P)")
    else:
        blocks = _batch_blocks()
        mine = batch_assignment(blocks, ws)[rank]
        entries, fs_total = [], 0
        for i, (cells, nv, order, scheme) in enumerate(blocks):
            m, n, p = (c - 1 for c in cells)
            gb = wsb.Grid(m, n, p, nv, BUFF, scheme=scheme)
            for d in range(3):
                ns, c1, c2 = gb.extents(d)
                fs_total += 2 * (ns if order == 3 else ns - 6) * c1 * c2 * nv
            if i not in mine:
                continue
            vb = fields.smooth_jump_field_dev(m, n, p, nv, BUFF, seed=100 + i, device=dev)
            for d in range(3):
                cf = tuple(torch.from_numpy(np.ascontiguousarray(c.ravel(order="F"))).to(dev)
                           for c in fields.uniform_weno_coefficients(order, gb.nc(d)))
                nface = int(np.prod(gb.face_shape(d)))
                entries.append(dict(grid=gb, dir=d, order=order, flags=wsb.F_MP | wsb.F_FOLDED, v_in=vb, coefs=cf,
                                    vL=torch.empty(nface, dtype=torch.float64, device=dev),
                                    vR=torch.empty(nface, dtype=torch.float64, device=dev)))
        b = api.Batch(entries)
        b.autotune(stream=sp)

        def step():
            b.launch(stream=sp)
        launches = 1
        workload = f"96 uneven blocks (x/y/z + MP each, FP64), LPT-placed over {ws} ranks ({len(mine)} here)"
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev.index if dev.index is not None else 0) as clk:
        e0.record(stream)
        for _ in range(K):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ms = e0.elapsed_time(e1) / K
    if dist is not None:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    if args.decomp == "batch":
        b.close()
    if rank == 0:
        print(json.dumps({
            "metric": METRIC if args.decomp == "zslab" else "batched face-states/s (96 uneven blocks, FP64)",
            "value": fs_total / (ms * 1e-3), "unit": "face-states/s", "n_gpus": ws, "steps": K,
            "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload, "decomp": args.decomp, "parallelism": f"{args.decomp} over {ws} ranks"},
            "gpu_launches": launches * K, "clocks": clk.summary()}), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def read_profile_value(key, kind=int):
    """A 'key: <number>' line of the committed ncu summary of the headline
    sweep (profiles/sweep_march_tma_fp64_200cubed.md), else None."""
    p = os.path.join(ROOT, "profiles", "sweep_march_tma_fp64_200cubed.md")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.strip().startswith(key + ":"):
                try:
                    return kind(line.split(":", 1)[1].strip().split()[0])
                except ValueError:
                    return None
    return None


def read_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (line 'traffic_bytes_per_launch: <int>'), else None."""
    return read_profile_value("traffic_bytes_per_launch", int)


def fp64_issue_bound(launch_ms, sm_mhz, sms=148):
    """The FP64-pipe bound of the headline sweep beside its HBM bound: the
    FP64 warp-instructions one launch issues (the measured count per warp
    and face of the committed ncu summary, times the launch's warp-faces:
    core faces x 32-column tiles x the other cross axis x variables), at
    half a warp-instruction per cycle per scheduler (4 per SM) and the SM
    clock seen during the timed region.  None without the summary."""
    per = read_profile_value("fp64_warp_inst_per_warp_face", float)
    if per is None or not sm_mhz:
        return None
    N = M + 2 * BUFF + 1
    NC = N - 6
    tiles = (N + 31) // 32
    inst = per * NC * tiles * N * NV
    floor_ms = inst * 2.0 / (sms * 4 * sm_mhz * 1e6) * 1e3
    return {"fp64_warp_inst_per_launch": inst, "fp64_warp_inst_per_warp_face": per, "sm_mhz": sm_mhz,
            "floor_ms": floor_ms, "launch_ms": launch_ms, "frac": floor_ms / launch_ms,
            "rule": "FP64 warp-instructions x 2 cycles / (148 SMs x 4 schedulers x SM clock)"}


def measure_fp32_bulk(g, v, faces, outs64, stream, K, dev):
    """FP32-bulk: FP32 sweep fields (reshaped from v_vf) and face states; FP64
    beta differences and weight normalisation.  Timed on the sweeps; error
    stated against the FP64 outputs of the same step (max-norm relative)."""
    import torch

    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import api
    sp = int(stream.cuda_stream)
    rs = [torch.empty(int(np.prod(g.rs_shape(d))), dtype=torch.float32, device=dev) for d in range(3)]
    nface = int(np.prod(g.face_shape(0)))
    o32 = [(torch.empty(nface, dtype=torch.float32, device=dev), torch.empty(nface, dtype=torch.float32, device=dev))
           for _ in range(3)]
    for d in range(3):
        api.reshape(g, d, v, rs[d], stream=sp)

    def step():
        for d in range(3):
            api.weno_uniform(g, d, ORDER, rs[d], faces[d], o32[d][0], o32[d][1], flags=wsb.F_MP, stream=sp)

    for _ in range(3):
        step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(K):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    # error vs the FP64 outputs of the folded FP64 step (core faces only)
    N = g.N[0]
    errs = []
    for d in range(3):
        for a64, a32 in zip(outs64[d], o32[d]):
            A = a64.view(NV, N, N, N)[:, :, :, 3:N - 3]
            B = a32.view(NV, N, N, N)[:, :, :, 3:N - 3].double()
            errs.append(float((A - B).abs().max() / A.abs().max()))
    fs = 3 * face_states_per_dir()
    return {"value": fs / (ms * 1e-3), "ms_per_step": ms, "max_rel_err_vs_fp64": max(errs),
            "data": "smooth-plus-jump (jump on odd variables)",
            "form": "drop-in (FP32 v_rs_ws, reshaped once outside the timed loop)"}


def measure_drop_in(g, v, faces, outs, stream, K, dev):
    """The drop-in form: s_initialize_weno (tiled-transpose reshape into
    v_rs_ws) then the sweep, per direction."""
    import torch

    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import api
    sp = int(stream.cuda_stream)
    rs = [torch.empty(int(np.prod(g.rs_shape(d))), dtype=torch.float64, device=dev) for d in range(3)]

    def step(reshape=True):
        for d in range(3):
            if reshape:
                api.reshape(g, d, v, rs[d], stream=sp)
            api.weno_uniform(g, d, ORDER, rs[d], faces[d], outs[d][0], outs[d][1], flags=wsb.F_MP, stream=sp)

    res = {}
    for reshape in (True, False):
        for _ in range(3):
            step(reshape)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(K):
            step(reshape)
        e1.record(stream)
        torch.cuda.synchronize()
        res["with_reshape_ms" if reshape else "sweeps_only_ms"] = e0.elapsed_time(e1) / K
    fs = 3 * face_states_per_dir()
    res["value_with_reshape"] = fs / (res["with_reshape_ms"] * 1e-3)
    res["value_sweeps_only"] = fs / (res["sweeps_only_ms"] * 1e-3)
    return res


def measure_e2e(g, vf_host, coefs, K, dev, full_download=False):
    """End to end through the C-ABI handle API (what a Fortran caller of the
    harness does): upload v_vf from pinned host memory (weno_sb_upload_async:
    the sweeps of each variable start once that variable has arrived), x/y/z
    folded WENO5 + MP, then read the step's result back to the host -- the
    harness's result
    is its checksum lines (f_checksum of each face-state array, f90:1617-1620,
    1836-1844), so by default the six checksums, summed on the device; with
    full_download the six face-state arrays themselves (3.66 GB) into pinned
    host memory.  Wall clock around each step."""
    import ctypes

    import torch

    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import _lib as L
    h = wsb.Harness(g)
    try:
        for d in range(3):
            h.upload_coefficients(d, [np.asarray(c.cpu().numpy()).reshape(s, order="F") for c, s in
                                      zip(coefs[d], [(g.nc(d), 5, 3), (g.nc(d), 5, 3), (5, g.nc(d)),
                                                     (5, g.nc(d)), (g.nc(d), 5, 6)])])
        src = torch.from_numpy(vf_host.ravel(order="F")).pin_memory()
        nface = int(np.prod(g.face_shape(0)))
        dst = [torch.empty(nface, dtype=torch.float64).pin_memory() for _ in range(6)] if full_download else []
        sums = [ctypes.c_double() for _ in range(6)]
        lib = L.lib()

        def step():
            # the copy runs one variable at a time and each folded sweep
            # waits only for its own variable (weno_sb_upload_async)
            L.check(lib.weno_sb_upload_async(h.handle, L.A_V_VF, src.data_ptr()))
            for d in range(3):
                L.check(lib.weno_sb_weno(h.handle, d, 5, wsb.F_MP | wsb.F_FOLDED))
            for d in range(3):
                if full_download:
                    L.check(lib.weno_sb_download(h.handle, L.A_VL(d), dst[2 * d].data_ptr()))
                    L.check(lib.weno_sb_download(h.handle, L.A_VR(d), dst[2 * d + 1].data_ptr()))
                else:
                    L.check(lib.weno_sb_checksum(h.handle, L.A_VL(d), ctypes.byref(sums[2 * d])))
                    L.check(lib.weno_sb_checksum(h.handle, L.A_VR(d), ctypes.byref(sums[2 * d + 1])))

        step()
        t0 = time.perf_counter()
        for _ in range(K):
            step()
        dt = (time.perf_counter() - t0) / K
    finally:
        h.close()
    fs = 3 * face_states_per_dir()
    out = {"value": fs / dt, "unit": "face-states/s", "h2d_bytes_per_step": int(vf_host.nbytes),
           "d2h_bytes_per_step": int(6 * nface * 8) if full_download else 6 * 8, "ms_per_step": dt * 1e3,
           "steps": K}
    out["path"] = ("weno_sb_upload_async (per-variable copies, each sweep waits for its variable) -> "
                   "weno_sb_weno x3 (folded, MP) -> " +
                   ("weno_sb_download x6 (all face states), pinned host buffers" if full_download else
                    "weno_sb_checksum x6 (the harness's result: f_checksum of every face-state array)"))
    return out


def _time_steps(step, stream, K, warm=3):
    """Mean device time of `step` over K calls (CUDA events on `stream`)."""
    import torch
    for _ in range(warm):
        step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(K):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / K


def measure_adjoint(dev, K):
    """Adjoint of FP64 WENO5-JS + MP in x/y/z at 128^3 cells x 5 variables:
    forward = three folded sweeps; backward = three VJP sweeps accumulating
    the gradient of v_vf (beta and the weights recomputed, nothing stored).
    Cotangents N(0,1) from a seeded generator; smooth sinusoidal input."""
    import torch

    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import api, fields
    m, nv = 127, 5
    g = wsb.Grid(m, m, m, nv, BUFF)
    stream = torch.cuda.Stream(device=dev)
    sp = int(stream.cuda_stream)
    v = fields.sinusoid_shock_field_dev(m, m, m, nv, BUFF, seed=4, shock=False, device=dev)
    faces = [api.face_coefs(fields.uniform_weno_coefficients(5, g.nc(d))) for d in range(3)]
    nface = int(np.prod(g.face_shape(0)))
    gen = torch.Generator(device=dev).manual_seed(8)
    gs = [(torch.randn(nface, generator=gen, device=dev, dtype=torch.float64),
           torch.randn(nface, generator=gen, device=dev, dtype=torch.float64)) for _ in range(3)]
    outs = (torch.empty(nface, dtype=torch.float64, device=dev), torch.empty(nface, dtype=torch.float64, device=dev))
    gv = torch.empty_like(v)
    fl = wsb.F_MP | wsb.F_FOLDED

    def fwd():
        for d in range(3):
            api.weno_uniform(g, d, 5, v, faces[d], outs[0], outs[1], flags=fl, stream=sp)

    def bwd():
        for d in range(3):
            api.vjp(g, d, 5, v, faces[d], gs[d][0], gs[d][1], gv, stream=sp, uniform=True,
                    flags=fl | (wsb.F_ACCUMULATE if d > 0 else 0))

    f_ms = _time_steps(fwd, stream, K)
    b_ms = _time_steps(bwd, stream, K)
    # the other families the adjoint covers (JS and TENO weights): forward
    # and VJP of the same step
    fam = {}
    for name, order, scheme, arrays in (("weno3_js", 3, wsb.JS, False), ("weno7_js", 7, wsb.JS, False),
                                        ("weno5_teno", 5, wsb.TENO, False), ("weno7_teno", 7, wsb.TENO, False),
                                        ("weno5_js_per_face_arrays", 5, wsb.JS, True)):
        gf = wsb.Grid(m, m, m, nv, BUFF, scheme=scheme)
        if arrays:
            # (the device tensors stay referenced while their pointers are used)
            held = [tuple(torch.from_numpy(np.ascontiguousarray(c.ravel(order="F"))).to(dev)
                          for c in fields.uniform_weno_coefficients(order, g.nc(d))) for d in range(3)]
            cf = held
        else:
            cf = [api.face_coefs(fields.uniform_weno_coefficients(order, g.nc(d))) for d in range(3)]

        def fwd_f(gf=gf, cf=cf, order=order, arrays=arrays):
            for d in range(3):
                if arrays:
                    api.weno(gf, d, order, v, cf[d], outs[0], outs[1], flags=fl, stream=sp)
                else:
                    api.weno_uniform(gf, d, order, v, cf[d], outs[0], outs[1], flags=fl, stream=sp)

        def bwd_f(gf=gf, cf=cf, order=order, arrays=arrays):
            for d in range(3):
                api.vjp(gf, d, order, v, cf[d], gs[d][0], gs[d][1], gv, stream=sp, uniform=not arrays,
                        flags=fl | (wsb.F_ACCUMULATE if d > 0 else 0))

        ff = _time_steps(fwd_f, stream, K)
        bb = _time_steps(bwd_f, stream, K)
        fam[name] = {"forward_ms": ff, "vjp_ms": bb, "vjp_over_forward": bb / ff}
    return {"workload": "VJP of FP64 WENO5-JS + MP, x/y/z, 128^3 cells x 5 vars, folded input, "
                        "uniform coefficients, cotangents N(0,1)",
            "forward_ms": f_ms, "vjp_ms": b_ms, "vjp_over_forward": b_ms / f_ms, "target_ratio": 2.5,
            "families": fam}


def _batch_blocks(n_blocks=96, seed=96):
    """Block shapes of the batched workload: cells per axis uniform in
    16..112, v_size from {5, 8, 10}, order from {3, 5, 7}, JS or TENO."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_blocks):
        cells = [int(c) for c in rng.integers(16, 113, 3)]
        nv = int(rng.choice([5, 8, 10]))
        order = int(rng.choice([3, 5, 7]))
        scheme = 0 if order == 3 else int(rng.choice([0, 3]))
        out.append((cells, nv, order, scheme))
    return out


def measure_batched(dev, K, n_blocks=96, layout=None, dtypes=("fp64", "fp32")):
    """96 uneven blocks (x/y/z sweeps each, MP fused, folded input) as one
    CUDA graph launch, run the way the autotuner picks (one persistent
    kernel over all blocks; per-block specialised sweeps on parallel graph
    branches; or grouped TMA marching sweeps, one launch per kernel
    instance over all its blocks), FP64 and FP32-bulk; the other ways and,
    FP64, one launch per sweep for comparison.  n_blocks < 96 takes the
    first blocks of the list; layout = (mode, threads, cols_per_item,
    branches) fixes the way instead of autotuning and skips the comparisons
    (a short command for profiling one way's kernels)."""
    import torch

    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import api, fields
    stream = torch.cuda.Stream(device=dev)
    sp = int(stream.cuda_stream)
    blocks = _batch_blocks()[:n_blocks]
    res = {"workload": "96 blocks, cells per axis U{16..112}, v_size {5,8,10}, order {3,5,7}, JS/TENO "
                       "(teno_CT 1e-5), smooth-plus-jump fields, x/y/z sweeps + MP each = 288 sweeps",
           "blocks": len(blocks)}
    for dt_name, dt in (("fp64", torch.float64), ("fp32", torch.float32)):
        if dt_name not in dtypes:
            continue
        entries, fs = [], 0
        for i, (cells, nv, order, scheme) in enumerate(blocks):
            m, n, p = (c - 1 for c in cells)
            g = wsb.Grid(m, n, p, nv, BUFF, scheme=scheme)
            v = fields.smooth_jump_field_dev(m, n, p, nv, BUFF, seed=100 + i, device=dev).to(dt)
            for d in range(3):
                cf = tuple(torch.from_numpy(np.ascontiguousarray(c.ravel(order="F"))).to(dev)
                           for c in fields.uniform_weno_coefficients(order, g.nc(d)))
                nface = int(np.prod(g.face_shape(d)))
                L = torch.empty(nface, dtype=dt, device=dev)
                R = torch.empty(nface, dtype=dt, device=dev)
                entries.append(dict(grid=g, dir=d, order=order, flags=wsb.F_MP | wsb.F_FOLDED, v_in=v,
                                    coefs=cf, vL=L, vR=R))
                ns, c1, c2 = g.extents(d)
                nf = ns if order == 3 else ns - 6
                fs += 2 * nf * c1 * c2 * nv
        b = api.Batch(entries)
        try:
            if layout is None:
                t, u, tune_ms = b.autotune(stream=sp)
            else:
                b.configure(*layout)
                t, u = layout[1], layout[2]
            mode, _, per_item, nb = b.query()
            ms = _time_steps(lambda: b.launch(stream=sp), stream, K)
            # the other ways of running the batch, at their default layouts
            other = {}
            for m_o, cfg, key in ((0, (0, 128, 8, 8), "persistent_kernel_ms"),
                                  (1, (1, 128, 8, 8), "graph_of_sweeps_8_branches_ms"),
                                  (2, (2, 128, 64, 2), "grouped_sweeps_64_faces_2_branches_ms")):
                if m_o != mode and layout is None:
                    b.configure(*cfg)
                    other[key] = _time_steps(lambda: b.launch(stream=sp), stream, K)
        finally:
            b.close()
        choice = {0: {"mode": "persistent kernel", "threads": t, "cols": u},
                  1: {"mode": "graph of specialised sweeps", "branches": nb},
                  2: {"mode": "grouped TMA marching sweeps", "faces_per_item": per_item, "branches": nb}}[mode]
        r = {"ms_per_step": ms, "value": fs / (ms * 1e-3), "face_states": fs, "choice": choice,
             "graph_launches_per_step": 1, **other}
        if dt == torch.float64 and layout is None:
            structs = [api.coefs_struct(e["coefs"]) for e in entries]

            def seq():
                for e, cs in zip(entries, structs):
                    api.weno(e["grid"], e["dir"], e["order"], e["v_in"], cs, e["vL"], e["vR"],
                             flags=e["flags"], stream=sp)
            sms = _time_steps(seq, stream, K)
            r["one_launch_per_sweep"] = {"ms_per_step": sms, "value": fs / (sms * 1e-3),
                                         "launches_per_step": len(entries)}
        res[dt_name] = r
        del entries
    return res


def measure_families(g, v, stream, K, dev):
    """Every kernel family of the path at 200^3 x 8 (FP64, x/y/z each):
    reshape (s_initialize_weno), order-1 copy, WENO3 / WENO5 / WENO7 with
    JS weights and MP fused, the standalone MP limiter, and WENO5 with TENO
    (teno_CT 1e-5), mapped and Z weights.  True uniform-grid coefficients go through the
    face-independent entry (weno_sb_weno_uniform_dev, which the handle API
    also takes when its coefficient banks are uniform); the harness's
    coefficient arrays (s_fill_coefficients) through the per-face entry
    (weno_sb_weno_dev), for WENO5 and WENO7.  ms per three sweeps."""
    import torch

    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import api, fields
    sp = int(stream.cuda_stream)
    nface = int(np.prod(g.face_shape(0)))
    L = torch.empty(nface, dtype=torch.float64, device=dev)
    R = torch.empty(nface, dtype=torch.float64, device=dev)
    rs = [torch.empty(int(np.prod(g.rs_shape(d))), dtype=torch.float64, device=dev) for d in range(3)]
    for d in range(3):
        api.reshape(g, d, v, rs[d], stream=sp)
    gt = wsb.Grid(M, M, M, NV, BUFF, scheme=wsb.TENO)
    res = {}

    def coefs(order, d, harness=False):
        c = (fields.harness_coefficients(g.nc(d), (0.03, 0.05, 0.07)[d]) if harness
             else fields.uniform_weno_coefficients(order, g.nc(d)))
        return tuple(torch.from_numpy(np.ascontiguousarray(x.ravel(order="F"))).to(dev) for x in c)

    def timed(name, fn):
        res[name] = {"ms_per_step": _time_steps(fn, stream, K)}
        res[name]["value"] = 3 * face_states_per_dir() / (res[name]["ms_per_step"] * 1e-3)

    timed("reshape", lambda: [api.reshape(g, d, v, rs[d], stream=sp) for d in range(3)])
    timed("order1_copy", lambda: [api.order1_copy(g, d, v, L, R, stream=sp) for d in range(3)])
    def face(order, d):
        return api.face_coefs(fields.uniform_weno_coefficients(order, g.nc(d)))

    for order in (3, 5, 7):
        fc = [face(order, d) for d in range(3)]
        timed(f"weno{order}_js_mp", lambda fc=fc, order=order: [
            api.weno_uniform(g, d, order, v, fc[d], L, R, flags=wsb.F_MP | wsb.F_FOLDED, stream=sp)
            for d in range(3)])
    for order in (5, 7):
        hc = [coefs(order, d, harness=True) for d in range(3)]
        timed(f"weno{order}_js_mp_harness_coefficient_arrays", lambda hc=hc, order=order: [
            api.weno(g, d, order, v, hc[d], L, R, flags=wsb.F_MP | wsb.F_FOLDED, stream=sp) for d in range(3)])
    timed("mp_standalone", lambda: [api.preserve_monotonicity(g, d, rs[d], L, R, stream=sp) for d in range(3)])
    fc5 = [face(5, d) for d in range(3)]
    timed("weno5_teno_mp", lambda: [
        api.weno_uniform(gt, d, 5, v, fc5[d], L, R, flags=wsb.F_MP | wsb.F_FOLDED, stream=sp) for d in range(3)])
    for name, scheme in (("weno5_mapped_mp", wsb.MAPPED), ("weno5_z_mp", wsb.Z)):
        gs = wsb.Grid(M, M, M, NV, BUFF, scheme=scheme)
        timed(name, lambda gs=gs: [
            api.weno_uniform(gs, d, 5, v, fc5[d], L, R, flags=wsb.F_MP | wsb.F_FOLDED, stream=sp) for d in range(3)])
    res["note"] = ("value = face-states/s of the WENO5 face count (3 x 148,135,424) for every family, so "
                   "the rows compare as times; WENO3 writes all ns faces")
    return res


def measure_mixed_precision(dev, K):
    """FP32-bulk against FP64 on 256^3 cells x 10 variables: WENO5 and WENO7
    + MP in x/y/z, FP32 fields (FP64-generated sinusoids, modes 1-8, plus a
    planar shock of jump ratio 5 at a seeded orientation, downcast) and FP32
    face states.  Error per output array against the FP64 path (which the
    parity tests hold to 1e-12 of the oracle): max-norm relative and RMS
    relative over the core faces; smooth (no shock) and shocked data."""
    import torch

    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import api, fields
    m, nv = 255, 10
    g = wsb.Grid(m, m, m, nv, BUFF)
    stream = torch.cuda.Stream(device=dev)
    sp = int(stream.cuda_stream)
    nface = int(np.prod(g.face_shape(0)))
    ns = g.extents(0)[0]
    o64 = (torch.empty(nface, dtype=torch.float64, device=dev), torch.empty(nface, dtype=torch.float64, device=dev))
    o32 = (torch.empty(nface, dtype=torch.float32, device=dev), torch.empty(nface, dtype=torch.float32, device=dev))
    rs32 = torch.empty(int(np.prod(g.rs_shape(0))), dtype=torch.float32, device=dev)
    res = {"workload": "256^3 cells x 10 vars, x/y/z + MP, FP32 fields and face states vs FP64",
           "error_reference": "FP64 sweeps of the same inputs (held to 1e-12 of the oracle by the tests)"}
    for order in (5, 7):
        faces = [api.face_coefs(fields.uniform_weno_coefficients(order, g.nc(d))) for d in range(3)]
        for shock in (False, True):
            v = fields.sinusoid_shock_field_dev(m, m, m, nv, BUFF, seed=11, shock=shock, device=dev)
            arrays = {}
            for d in range(3):
                api.weno_uniform(g, d, order, v, faces[d], o64[0], o64[1], flags=wsb.F_MP | wsb.F_FOLDED, stream=sp)
                api.reshape(g, d, v, rs32, stream=sp)
                api.weno_uniform(g, d, order, rs32, faces[d], o32[0], o32[1], flags=wsb.F_MP, stream=sp)
                torch.cuda.synchronize()
                for nm, a, b in (("vL", o64[0], o32[0]), ("vR", o64[1], o32[1])):
                    A = a.view(-1, ns)[:, 3:ns - 3]
                    B = b.view(-1, ns)[:, 3:ns - 3].double()
                    den = float(A.abs().max())
                    diff = (A - B)
                    arrays[f"{nm}_{'xyz'[d]}"] = {
                        "max_rel": float(diff.abs().max()) / den,
                        "rms_rel": float(diff.pow(2).mean().sqrt() / A.pow(2).mean().sqrt())}
            res[f"weno{order}_{'shock' if shock else 'smooth'}"] = {
                "max_rel_worst": max(x["max_rel"] for x in arrays.values()),
                "rms_rel_worst": max(x["rms_rel"] for x in arrays.values()), "per_array": arrays}
            if not shock:
                def s64():
                    for d in range(3):
                        api.weno_uniform(g, d, order, v, faces[d], o64[0], o64[1],
                                         flags=wsb.F_MP | wsb.F_FOLDED, stream=sp)
                rsd = [torch.empty(int(np.prod(g.rs_shape(d))), dtype=torch.float32, device=dev) for d in range(3)]
                for d in range(3):
                    api.reshape(g, d, v, rsd[d], stream=sp)

                def s32():
                    for d in range(3):
                        api.weno_uniform(g, d, order, rsd[d], faces[d], o32[0], o32[1], flags=wsb.F_MP, stream=sp)
                t64 = _time_steps(s64, stream, K)
                t32 = _time_steps(s32, stream, K)
                fs = 3 * face_states_per_dir(m=m, nv=nv)
                res[f"weno{order}_speed"] = {"fp64_ms": t64, "fp32_ms": t32, "fp32_over_fp64": t64 / t32,
                                             "fp64_value": fs / (t64 * 1e-3), "fp32_value": fs / (t32 * 1e-3)}
                del rsd
            del v
    return res


def run_only(args):
    """One side measurement (the adjoint or the batched blocks) alone on
    cuda:0 with K = --steps timed steps: its result as one JSON line."""
    import torch
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    if args.only == "batched":
        layout = tuple(int(x) for x in args.batch_layout.split(",")) if args.batch_layout else None
        dtypes = ("fp64", "fp32") if args.batch_dtype == "both" else (args.batch_dtype,)
        res = measure_batched(dev, max(1, args.steps), n_blocks=args.batch_blocks, layout=layout, dtypes=dtypes)
    else:
        res = measure_adjoint(dev, max(1, args.steps))
    print(json.dumps({"measurement": args.only, **res}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-extras", action="store_true", help="skip FP32/drop-in/e2e side measurements")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--m", type=int, default=199, help="cells per axis minus one (m=n=p); 199 = 200^3")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64",
                    help="fp32: time the FP32-bulk form as the main step (no extras)")
    ap.add_argument("--order", type=int, choices=[3, 5, 7], default=5,
                    help="reconstruction order of the main step (5 is the headline metric; others skip the extras)")
    ap.add_argument("--scheme", choices=["js", "teno"], default="js",
                    help="nonlinear weights of the main step (teno: teno_CT 1e-5; WENO5 / WENO7 only)")
    ap.add_argument("--coefficients", choices=["uniform", "arrays", "stretched"], default="uniform",
                    help="arrays: the main step passes the uniform-grid coefficients as per-face device "
                         "arrays (weno_sb_weno_dev, the drop-in form) instead of one face-independent set; "
                         "stretched: per-face arrays of a tanh-stretched grid (weno_sb_coefficients)")
    ap.add_argument("--decomp", choices=["blocks", "zslab", "batch"], default="blocks",
                    help="blocks: one 200^3 x 8 block per rank (weak scaling, the default); zslab: one block "
                         "split along z with a ghost-plane exchange per step; batch: the 96-block batch placed "
                         "on the ranks by LPT (both strong scaling)")
    ap.add_argument("--only", choices=["adjoint", "batched"], default=None,
                    help="run only this side measurement on cuda:0 and print its JSON line "
                         "(a short command whose kernels can be profiled alone)")
    ap.add_argument("--batch-blocks", type=int, default=96,
                    help="--only batched: the first N blocks of the 96-block list")
    ap.add_argument("--batch-layout", default=None,
                    help="--only batched: MODE,THREADS,COLS_PER_ITEM,BRANCHES instead of autotuning "
                         "(no comparisons with the other ways)")
    ap.add_argument("--batch-dtype", choices=["fp64", "fp32", "both"], default="both",
                    help="--only batched: storage precisions to run")
    args = ap.parse_args()
    if args.only:
        return run_only(args)
    global M, ORDER, SCHEME
    M = args.m
    ORDER = args.order
    SCHEME = args.scheme
    if ORDER == 3 and SCHEME == "teno":
        ap.error("WENO3 has no TENO weights (f90:392-475)")
    if ORDER != 5 or SCHEME != "js":
        args.no_extras = True
    if args.impl == "reference":
        return run_reference(args)
    if args.decomp != "blocks":
        return run_decomp(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
