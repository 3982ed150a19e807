#!/usr/bin/env python
"""Benchmark of the HEVI short step (SCALE-RM ATMOS_DYN_Tstep_short_fvm_hevi) on B200.

Workload: the 512x512x128 configuration (dx = dy = 250 m, dz stretched 50 m to
400 m, CD4 momentum/scalar flux, dt = 0.5 s, three moist tracers with FCT),
synthetic seeded inputs (no public dataset is involved). One step is one
iteration of the short-step loop of the large step
(scale_atmos_dyn_tstep_large_fvm_heve.F90:600-944): the numerical filter
coefficients, the RK4 short step (four HEVI stages with their device halo
exchanges and the combine) and the boundary values + halo exchange of the
state. The metric is interior cell-updates per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun with N > 1 every rank runs its own replica of the workload on
its GPU (the path is single-GPU by specification; no data-path collective) and
the value is the aggregate over ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "HEVI short-step cell-updates/s on 1 B200, FP64 vs mixed at stated error; %HBM"
UNIT = "cell-updates/s"
L2_BYTES = 126 * 1024 * 1024
HEVE_DT = 0.04  # s; below the vertical acoustic limit dz / c_s of the 50 m lowest layer
# algorithmic bytes per interior cell: one HEVI stage reads 34
# fields (DENS0..RHOT0, DENS..RHOT, *_t, DPRES0, RT2P, REF_dens, REF_rhot and the
# 15 num_diff components; DDIV is not read because divdmp_coef = 0) and writes 11
# (DENS_RK..RHOT_RK, mflx_hi(3), tflx_hi(3)); the filter reads 7 and writes 15.
STAGE_BYTES = (34 + 11) * 8
NUMFILTER_BYTES = (7 + 15) * 8
STEP_BYTES = 4 * STAGE_BYTES + NUMFILTER_BYTES
# mixed precision: the 19 state and base-state fields stay FP64, the flux-like
# fields (num_diff 15, tendencies 5, mflx_hi 3, tflx_hi 3) are FP32
MIXED_STAGE_BYTES = (5 + 5 + 4) * 8 + 5 * 8 + (15 + 5 + 3 + 3) * 4
MIXED_NUMFILTER_BYTES = 7 * 8 + 15 * 4
# tracer advection, per tracer and large step: 3 RK stages, each reading QTRC,
# QTRC0, RHOQ_t, DENS0, DENS, mflx_hi (3) and the tracer num_diff (3) and
# writing QTRCo
TRACER_BYTES = 3 * 12 * 8


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def max_over_ranks(value: float, dist, device) -> float:
    """The slowest rank's time (every rank takes part; returns the local value
    without a process group)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: int, world: int, steps: int, elapsed_ms: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return world * units_per_rank * steps / (elapsed_ms * 1e-3)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.window = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"hevi_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def mark(self, t0: float, t1: float):
        """Host wall-clock bounds of the timed region."""
        self.window = (t0, t1)

    def summary(self):
        if self.proc is None or not self.path.exists():
            return None
        from datetime import datetime

        rows = []
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.path.read_text().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                ts = datetime.strptime(p[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(p[1]), float(p[2]), float(p[3]),
                             [n for n, v in zip(names, p[5:9]) if v.lower() == "active"]))
            except ValueError:
                continue
        self.path.unlink(missing_ok=True)
        inside = [r for r in rows if self.window and self.window[0] <= r[0] <= self.window[1]]
        used = inside or rows
        if not used:
            return None
        return {"sm_mhz": statistics.median(r[1] for r in used), "sm_max_mhz": used[-1][2],
                "power_w": statistics.median(r[3] for r in used),
                "reasons": sorted({n for r in used for n in r[4]}), "samples": len(used),
                "window": "timed region" if inside else "warm-up and timed region"}


# ---------------------------------------------------------------------------
# inputs
# ---------------------------------------------------------------------------
def make_inputs(scale: float):
    from scale_b200 import mkinit

    c = mkinit.config(2, scale=scale, seed=0)
    RT2P, DPRES0, REF_rhot = mkinit.large_prep(c)
    return c, RT2P, DPRES0, REF_rhot


def to_dev(x, torch):
    return torch.from_numpy(np.ravel(x, order="K")).cuda()


# ---------------------------------------------------------------------------
# the B200 arm
# ---------------------------------------------------------------------------
def run_b200(args):
    import torch

    from scale_b200 import hevi

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    c, RT2P, DPRES0, REF_rhot = make_inputs(args.scale)
    g = c.g
    N3 = int(np.prod(g.shape))
    cells = g.cells
    hevi.setup(g.index_dict(), c.scheme, c.scheme_tracer, device=local)
    if args.stage_shape:
        hevi.stage_shape(*[int(v) for v in args.stage_shape.split(",")])
    else:
        hevi.stage_autotune(True)  # the first warm-up step picks the stage tile shape

    # device-resident state and inputs (Fortran layout, one flat buffer each)
    st = torch.empty((5, N3), dtype=torch.float64, device="cuda")
    for v, n in enumerate(("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")):
        st[v].copy_(to_dev(c.state[n], torch))
    X = dict(DENS=st[0], MOMZ=st[1], MOMX=st[2], MOMY=st[3], RHOT=st[4])
    st0 = st.clone() if not (args.no_mixed and args.no_heve and args.no_terrain) else None
    z = lambda k=1: torch.zeros(k * N3, dtype=torch.float64, device="cuda")  # noqa: E731
    mflx, tflx, nd = z(3), z(3), z(15)
    tend = {n: z() for n in ("DENS_t", "MOMZ_t", "MOMX_t", "MOMY_t", "RHOT_t")}
    ref = {n: to_dev(v, torch) for n, v in c.ref.items()}
    dp0, rt2p, refr = to_dev(DPRES0, torch), to_dev(RT2P, torch), to_dev(REF_rhot, torch)
    GS = torch.ones(7 * N3, dtype=torch.float64, device="cuda")
    J0 = torch.zeros(7 * N3, dtype=torch.float64, device="cuda")
    MAPF = torch.ones(g.IA * g.JA * 8, dtype=torch.float64, device="cuda")
    cor = torch.zeros(g.IA * g.JA, dtype=torch.float64, device="cuda")
    wd = np.zeros(g.KA)
    grid = dict(CDZ=g.CDZ, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY, RFDZ=g.RFDZ,
                RFDX=g.RFDX, RFDY=g.RFDY)
    dts = c.dt

    def step(dts=dts, met=None):
        # met: (GSQRT, J13G, J23G, MAPF) device arrays of terrain-following metrics, or flat terrain
        gs, j13, j23, mp = met if met is not None else (GS, J0, J0, MAPF)
        # numerical filter (tstep_large:847-858) on the state at the start of the short step
        hevi.ATMOS_DYN_numfilter_coef_dev(num_diff=nd, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY, FDZ=g.FDZ, FDX=g.FDX,
                                          FDY=g.FDY, DT=dts, REF_dens=ref["REF_dens"], REF_pott=ref["REF_pott"],
                                          ND_COEF=c.nd_coef, ND_ORDER=1, ND_SFC_FACT=1.0, ND_USE_RS=True, **X)
        # RK4 short step (tstep_large:880-894)
        hevi.ATMOS_DYN_Tinteg_short_rk4_dev(
            PROG=None, mflx_hi=mflx, tflx_hi=tflx, DPRES0=dp0, RT2P=rt2p, CORIOLI=cor, num_diff=nd, wdamp_coef=wd,
            divdmp_coef=0.0, DDIV=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False, FLAG_FCT_ALONG_STREAM=True,
            PHI=ref["PHI"], GSQRT=gs, J13G=j13, J23G=j23, J33G=1.0, MAPF=mp, REF_dens=ref["REF_dens"],
            REF_rhot=refr, BND_W=False, BND_E=False, BND_S=False, BND_N=False, dt=dts, **X, **tend, **grid)
        # vertical boundary values + halo exchange of the state (tstep_large:910-944)
        hevi.boundary_dev(**X)

    stream = torch.cuda.ExternalStream(hevi.stream_handle())
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        # warm-up (also keeps the GPU loaded while the clock sampler starts)
        for _ in range(args.warmup):
            step()
        hevi.check()
        m0 = hevi.domain_sum_dev(X["DENS"], g.CDZ, g.CDX, g.CDY)
        e0 = hevi.energy_sum_dev(**X, CZ=g.CZ, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY)

        # ---- timed region ----
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        hevi.profile(True)
        launches0 = hevi.kernel_launches()
        w0 = time.time()
        t0.record(stream)
        for _ in range(args.steps):
            step()
        t1.record(stream)
        torch.cuda.synchronize()
        clk.mark(w0, time.time())
    launches = hevi.kernel_launches() - launches0
    prof = hevi.profile_report()
    hevi.profile(False)
    elapsed_ms = max_over_ranks(t0.elapsed_time(t1), dist, "cuda")
    hevi.check()
    m1 = hevi.domain_sum_dev(X["DENS"], g.CDZ, g.CDX, g.CDY)
    e1 = hevi.energy_sum_dev(**X, CZ=g.CZ, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY)
    clocks = clk.summary()
    ms_step = elapsed_ms / args.steps
    value = aggregate_rate(cells, world, args.steps, elapsed_ms)

    # ---- roofline of the HEVI stage (tiled: k_hevi_explicit + k_hevi_column) ----
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    nst, stage_total = prof.get("hevi_stage", (0, 0.0))
    stage_ms = stage_total / max(nst, 1)
    achieved = STAGE_BYTES * cells / (stage_ms * 1e-3) / 1e9 if stage_ms > 0 else None
    traffic = read_traffic()
    roofline = {"bound": "hbm", "kernel": stage_form_name(hevi),
                "achieved": achieved, "peak": hbm, "peak_source": peak_src, "unit": "GB/s",
                "frac": (achieved / hbm) if achieved else None, "algorithmic_bytes_per_launch": STAGE_BYTES * cells,
                "stage_ms": stage_ms, "traffic": traffic,
                "step_frac": STEP_BYTES * cells / (ms_step * 1e-3) / 1e9 / hbm}

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; no dataset involved)",
        "config": {"workload": f"{g.IMAX}x{g.JMAX}x{g.KMAX} stretched dz 50-400 m, dx=250 m, CD4, dt=0.5 s, "
                               "short step = numfilter + RK4 (4 HEVI stages) + boundary/halo",
                   "cells": cells, "scheme": c.scheme, "integrator": "RK4", "precision": "fp64 (plain)",
                   "l2": f"inputs larger than L2 ({N3 * 8 / 2**20:.0f} MiB per field > {L2_BYTES / 2**20:.0f} MiB)",
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "roofline": roofline,
        "sections_ms_per_step": {k: v[1] / args.steps for k, v in prof.items()},
        "mass_drift_rel": abs(m1 - m0) / m0,
        "energy_budget": {"unit": "J", "before": e0, "after": e1,
                          "ENGT_change_rel": (e1["ENGT"] - e0["ENGT"]) / e0["ENGT"],
                          "sum": "FP64, on the device, fixed order (scale_hevi_energy_sum_dev)"},
        "gpu_launches": launches,
        "clocks": clocks,
        "autotune": hevi.autotune_report(),
    }

    if not args.no_mixed:
        # the same workload from the same initial state on the mixed-precision path
        st_fp64 = st.clone()
        st.copy_(st0)
        f32 = lambda k=1: torch.zeros(k * N3, dtype=torch.float32, device="cuda")  # noqa: E731
        mflx32, tflx32, nd32 = f32(3), f32(3), f32(15)
        tend32 = {n: f32() for n in ("DENS_t", "MOMZ_t", "MOMX_t", "MOMY_t", "RHOT_t")}

        def step_mixed():
            hevi.ATMOS_DYN_numfilter_coef_mixed_dev(num_diff=nd32, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY, FDZ=g.FDZ,
                                                    FDX=g.FDX, FDY=g.FDY, DT=dts, REF_dens=ref["REF_dens"],
                                                    REF_pott=ref["REF_pott"], ND_COEF=c.nd_coef, ND_ORDER=1,
                                                    ND_SFC_FACT=1.0, ND_USE_RS=True, **X)
            hevi.ATMOS_DYN_Tinteg_short_rk4_mixed_dev(
                PROG=None, mflx_hi=mflx32, tflx_hi=tflx32, DPRES0=dp0, RT2P=rt2p, CORIOLI=cor, num_diff=nd32,
                wdamp_coef=wd, divdmp_coef=0.0, DDIV=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False,
                FLAG_FCT_ALONG_STREAM=True, PHI=ref["PHI"], GSQRT=GS, J13G=J0, J23G=J0, J33G=1.0, MAPF=MAPF,
                REF_dens=ref["REF_dens"], REF_rhot=refr, BND_W=False, BND_E=False, BND_S=False, BND_N=False,
                dt=dts, **X, **tend32, **grid)
            hevi.boundary_dev(**X)

        for _ in range(args.warmup):
            step_mixed()
        hevi.check()
        m0x = hevi.domain_sum_dev(X["DENS"], g.CDZ, g.CDX, g.CDY)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        hevi.profile(True)
        t0.record(stream)
        for _ in range(args.steps):
            step_mixed()
        t1.record(stream)
        torch.cuda.synchronize()
        profm = hevi.profile_report()
        hevi.profile(False)
        hevi.check()
        m1x = hevi.domain_sum_dev(X["DENS"], g.CDZ, g.CDX, g.CDY)
        e_mixed = hevi.energy_sum_dev(**X, CZ=g.CZ, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY)
        ms_mixed = max_over_ranks(t0.elapsed_time(t1), dist, "cuda") / args.steps
        nsm, tsm = profm.get("hevi_stage_mixed", (0, 0.0))
        sm_ms = tsm / max(nsm, 1)
        ach = MIXED_STAGE_BYTES * cells / (sm_ms * 1e-3) / 1e9 if sm_ms > 0 else None
        # error of the mixed state against the FP64 state after the same steps,
        # relative to each field's largest magnitude over the interior
        sl = (slice(g.KS - 1, g.KE), slice(g.IS - 1, g.IE), slice(g.JS - 1, g.JE))
        errs = {}
        for v, n in enumerate(("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")):
            a64 = st_fp64[v].view(g.JA, g.IA, g.KA).permute(2, 1, 0)[sl[0], sl[1], sl[2]]
            a32 = st[v].view(g.JA, g.IA, g.KA).permute(2, 1, 0)[sl[0], sl[1], sl[2]]
            d = (a32 - a64).abs()
            scale = float(a64.abs().max())
            errs[n] = {"max": float(d.max()) / scale, "rms": float(d.pow(2).mean().sqrt()) / scale}
        out["mixed"] = {
            "value": aggregate_rate(cells, world, 1, ms_mixed), "unit": UNIT, "ms_per_step": ms_mixed,
            "speedup_vs_fp64": ms_step / ms_mixed,
            "precision": "FP32 flux and divergence arithmetic and FP32 num_diff/tendency/flux arrays; FP64 state, "
                         "base-state deviations, right-hand side and tridiagonal solve",
            "error_vs_fp64": {"steps": args.warmup + args.steps, "fields": errs},
            "mass_drift_rel": abs(m1x - m0x) / m0x,
            "energy_ENGT_vs_fp64_rel": (e_mixed["ENGT"] - e1["ENGT"]) / e1["ENGT"],
            "roofline": {"bound": "hbm", "kernel": stage_form_name(hevi, "float"), "achieved": ach,
                         "peak": hbm, "unit": "GB/s", "frac": (ach / hbm) if ach else None,
                         "algorithmic_bytes_per_launch": MIXED_STAGE_BYTES * cells, "stage_ms": sm_ms,
                         "step_frac": (4 * MIXED_STAGE_BYTES + MIXED_NUMFILTER_BYTES) * cells / (ms_mixed * 1e-3) / 1e9 / hbm},
            "sections_ms_per_step": {k: v[1] / args.steps for k, v in profm.items()},
        }
        del st_fp64

    if not args.no_tracer:
        out["tracer"] = run_tracer(args, c, hevi, torch, X, mflx, g, cells, stream, t0, t1, dist, world, hbm)
    if not args.no_heve:
        out["heve"] = run_heve(args, hevi, torch, step, st, st0, X, g, cells, stream, t0, t1, dist, world, hbm)
    if not args.no_terrain:
        out["terrain"] = run_terrain(args, hevi, torch, step, st, st0, g, cells, stream, t0, t1, dist, world, hbm)
    del st0

    if rank == 0 and not args.no_e2e:
        out["e2e"] = run_e2e(args, c, hevi, torch)
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args)
    hevi.finalize()
    if world == 1 and not (args.no_ensemble and args.no_mixed_large):
        del st, X, mflx, tflx, nd, tend, ref, dp0, rt2p, refr, GS, J0, MAPF, cor
        torch.cuda.empty_cache()
    if world == 1 and not args.no_mixed_large:
        out["mixed_1024x1024x96"] = run_mixed_large(args, hevi, torch)
        torch.cuda.empty_cache()
    if world == 1 and not args.no_ensemble:
        out["ensemble"] = run_ensemble(args, hevi, torch)
    if world == 1 and not args.no_adjoint:
        out["adjoint"] = run_adjoint(args, hevi, torch)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_heve(args, hevi, torch, step, st, st0, X, g, cells, stream, t0, t1, dist, world, hbm):
    """The same short steps with HEVE registered as the short step
    (ATMOS_DYN_Tstep_short_fvm_heve, explicit in the vertical too), from the
    same initial state. HEVE's step is bounded by the vertical acoustic limit
    dz / c_s of the 50 m lowest layer, so it runs at dt = 0.04 s; the work
    per step does not depend on dt."""
    st.copy_(st0)
    hevi.short_type("HEVE")
    try:
        for _ in range(args.warmup):
            step(HEVE_DT)
        hevi.check()
        m0 = hevi.domain_sum_dev(X["DENS"], g.CDZ, g.CDX, g.CDY)
        e0 = hevi.energy_sum_dev(**X, CZ=g.CZ, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        hevi.profile(True)
        t0.record(stream)
        for _ in range(args.steps):
            step(HEVE_DT)
        t1.record(stream)
        torch.cuda.synchronize()
        prof = hevi.profile_report()
        hevi.profile(False)
        hevi.check()
        m1 = hevi.domain_sum_dev(X["DENS"], g.CDZ, g.CDX, g.CDY)
    finally:
        hevi.short_type("HEVI")
    ms = max_over_ranks(t0.elapsed_time(t1), dist, "cuda") / args.steps
    n, tot = prof.get("heve_stage", (0, 0.0))
    stage_ms = tot / max(n, 1)
    ach = STAGE_BYTES * cells / (stage_ms * 1e-3) / 1e9 if stage_ms > 0 else None
    return {
        "value": aggregate_rate(cells, world, 1, ms), "unit": UNIT, "ms_per_step": ms, "dt": HEVE_DT,
        "step": "numfilter + RK4 of 4 HEVE stages + boundary/halo, FP64, same workload",
        "mass_drift_rel": abs(m1 - m0) / m0,
        "roofline": {"bound": "hbm", "kernel": "k_heve_stage (one HEVE stage)", "achieved": ach, "peak": hbm,
                     "unit": "GB/s", "frac": (ach / hbm) if ach else None,
                     "algorithmic_bytes_per_launch": STAGE_BYTES * cells, "stage_ms": stage_ms},
        "sections_ms_per_step": {k: v[1] / args.steps for k, v in prof.items()},
    }


TERRAIN_STEPS = 10  # timed steps of the terrain leg (about 0.9 s of work)
TERRAIN_BYTES = STAGE_BYTES + 15 * 8  # the flat stage's bytes plus 15 metric slices per cell


def terrain_metrics(g, torch):
    """Smooth, periodic terrain-following metrics on the device: GSQRT and MAPF
    within 2% and 1% of 1, J13G and J23G within 0.01 of 0, the same at every
    staggering (seeded by nothing: a fixed analytic field)."""
    import numpy as np

    x = 2 * np.pi * (np.arange(g.IA) - (g.IS - 1)) / g.IMAX
    y = 2 * np.pi * (np.arange(g.JA) - (g.JS - 1)) / g.JMAX
    zf = np.linspace(1.0, 0.0, g.KA)[:, None, None]
    h = np.sin(x)[None, :, None] * np.sin(y)[None, None, :]
    gs = (1.0 + 0.02 * h * zf).ravel(order="F")
    j13 = (0.01 * np.cos(x)[None, :, None] * np.sin(y)[None, None, :] * zf).ravel(order="F")
    j23 = (0.01 * np.sin(x)[None, :, None] * np.cos(y)[None, None, :] * zf).ravel(order="F")
    m = (1.0 + 0.01 * np.sin(x)[:, None] * np.cos(y)[None, :]).ravel(order="F")
    dev = lambda a, n: torch.from_numpy(np.tile(a, n)).cuda()  # noqa: E731
    return dev(gs, 7), dev(j13, 7), dev(j23, 7), dev(m, 8)


def run_terrain(args, hevi, torch, step, st, st0, g, cells, stream, t0, t1, dist, world, hbm):
    """The same short steps with terrain-following metrics: the general-metric
    HEVI stage (one launch per loop nest of the reference) in place of the
    fused flat-terrain kernel, from the same initial state."""
    st.copy_(st0)
    met = terrain_metrics(g, torch)
    for _ in range(args.warmup):
        step(met=met)
    hevi.check()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    hevi.profile(True)
    t0.record(stream)
    for _ in range(TERRAIN_STEPS):
        step(met=met)
    t1.record(stream)
    torch.cuda.synchronize()
    prof = hevi.profile_report()
    hevi.profile(False)
    hevi.check()
    ms = max_over_ranks(t0.elapsed_time(t1), dist, "cuda") / TERRAIN_STEPS
    n, tot = prof.get("hevi_stage_terrain", (0, 0.0))
    stage_ms = tot / max(n, 1)
    ach = TERRAIN_BYTES * cells / (stage_ms * 1e-3) / 1e9 if stage_ms > 0 else None
    return {
        "value": aggregate_rate(cells, world, 1, ms), "unit": UNIT, "ms_per_step": ms, "steps": TERRAIN_STEPS,
        "step": "numfilter + RK4 of 4 general-metric HEVI stages + boundary/halo, FP64, same workload, smooth "
                "periodic metrics (GSQRT, MAPF within 2%/1% of 1; J13G, J23G within 0.01)",
        "roofline": {"bound": "hbm", "kernel": "terrain_stage (26 launches, one HEVI stage)", "achieved": ach,
                     "peak": hbm, "unit": "GB/s", "frac": (ach / hbm) if ach else None,
                     "algorithmic_bytes_per_launch": TERRAIN_BYTES * cells, "stage_ms": stage_ms},
        "sections_ms_per_step": {k: v[1] / TERRAIN_STEPS for k, v in prof.items()},
    }


def run_tracer(args, c, hevi, torch, X, mflx, g, cells, stream, t0, t1, dist, world, hbm):
    """Tracer advection of the workload's three moist tracers (QV at 80 % RH,
    QC = QR = 0) over one large step each: ATMOS_DYN_Tinteg_tracer_rk3_b200_dev
    (RK3WS2002, UD3 fluxes, FCT along-stream in the last stage), FP64, with the
    mass fluxes of the last short step and a tracer num_diff array, timed on
    the library stream. Algorithmic bytes: 11 fields read and 1 written per
    cell and RK stage, 3 stages: 288 B per cell per tracer and large step."""
    N3 = int(np.prod(g.shape))
    q0 = torch.from_numpy(np.ravel(c.state["QTRC"], order="K").copy()).cuda()  # (KA,IA,JA,3)
    qt = q0.clone()
    q_start = [q0[n * N3:(n + 1) * N3].clone() for n in range(c.QA)]
    zero = torch.zeros(N3, dtype=torch.float64, device="cuda")
    ndq = torch.zeros(3 * N3, dtype=torch.float64, device="cuda")
    dens0 = X["DENS"].clone()
    kw = dict(RHOQ_t=zero, DENS0=dens0, DENS=X["DENS"], mflx_hi=mflx, num_diff=ndq, GSQRT=None, MAPF=None,
              CDZ=g.CDZ, RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY, BND_W=False, BND_E=False, BND_S=False, BND_N=False,
              dtl=c.dtl, FLAG_FCT_TRACER=True, FLAG_FCT_ALONG_STREAM=True)

    def large_step():
        for n in range(c.QA):
            qn = qt[n * N3:(n + 1) * N3]
            hevi.ATMOS_DYN_Tinteg_tracer_rk3_dev(QTRC=qn, QTRC0=qn, **kw)

    k = max(1, args.tracer_steps)
    for _ in range(max(3, args.warmup)):
        large_step()
    hevi.check()
    qt.copy_(q0)
    torch.cuda.synchronize()
    hevi.profile(True)
    l0 = hevi.kernel_launches()
    t0.record(stream)
    for _ in range(k):
        large_step()
    t1.record(stream)
    torch.cuda.synchronize()
    prof = hevi.profile_report()
    hevi.profile(False)
    hevi.check()
    launches = hevi.kernel_launches() - l0
    ms = max_over_ranks(t0.elapsed_time(t1), dist, "cuda") / k
    ms_tracer = ms / c.QA
    ach = TRACER_BYTES * cells / (ms_tracer * 1e-3) / 1e9
    qmin = min(float(qt[n * N3:(n + 1) * N3].min()) for n in range(c.QA))
    # tracer mass (rho*q) after the steps against the start, FP64 device sums
    rq = [hevi.domain_sum_dev(X["DENS"] * qt[n * N3:(n + 1) * N3], g.CDZ, g.CDX, g.CDY) for n in range(c.QA)]
    rq0 = [hevi.domain_sum_dev(dens0 * q_start[n], g.CDZ, g.CDX, g.CDY) for n in range(c.QA)]

    # the same large steps with the three-kernel limiter (phi_lo and the
    # anti-diffusive fluxes through HBM), from the same start: its time, and
    # the fused form's result against it (identical bits expected)
    q64 = qt.clone()
    hevi.tracer_fct_form(False)
    try:
        qt.copy_(q0)
        torch.cuda.synchronize()
        t0.record(stream)
        for _ in range(k):
            large_step()
        t1.record(stream)
        torch.cuda.synchronize()
        hevi.check()
    finally:
        hevi.tracer_fct_form(True)
    ms3 = max_over_ranks(t0.elapsed_time(t1), dist, "cuda") / k / c.QA
    three_kernel = {"ms_per_tracer_large_step": ms3, "fused_speedup": ms3 / ms_tracer,
                    "fused_result_identical": bool(torch.equal(qt, q64))}
    qt.copy_(q64)

    # the same large steps with FP32 flux and limiter arithmetic, from the same start
    kw32 = dict(kw, RHOQ_t=zero.float(), mflx_hi=mflx.float(), num_diff=ndq.float())

    def large_step_mixed():
        for n in range(c.QA):
            qn = qt[n * N3:(n + 1) * N3]
            hevi.ATMOS_DYN_Tinteg_tracer_rk3_mixed_dev(QTRC=qn, QTRC0=qn, **kw32)

    for _ in range(max(3, args.warmup)):
        large_step_mixed()
    hevi.check()
    qt.copy_(q0)
    torch.cuda.synchronize()
    t0.record(stream)
    for _ in range(k):
        large_step_mixed()
    t1.record(stream)
    torch.cuda.synchronize()
    hevi.check()
    ms32 = max_over_ranks(t0.elapsed_time(t1), dist, "cuda") / k / c.QA
    err32 = float((qt - q64).abs().max()) / float(q64.abs().max())
    mixed = {"ms_per_tracer_large_step": ms32, "speedup_vs_fp64": ms_tracer / ms32,
             "precision": "FP32 flux and FCT limiter arithmetic, FP32 mass fluxes, num_diff and tendency; FP64 tracer, "
                          "densities and update",
             "max_rel_error_vs_fp64": err32, "large_steps": k,
             "min_tracer_after": min(float(qt[n * N3:(n + 1) * N3].min()) for n in range(c.QA))}
    return {
        "value": aggregate_rate(cells, world, 1, ms_tracer), "unit": "cell-updates/s per tracer",
        "ms_per_tracer_large_step": ms_tracer, "ms_per_large_step": ms, "tracers": c.QA, "large_steps": k,
        "step": "ATMOS_DYN_Tinteg_tracer_rk3 (3 RK stages, UD3 fluxes, FCT along-stream), dtl = 2.5 s, FP64",
        "roofline": {"bound": "hbm", "kernel": "tracer RK3 with FCT (k_tracer_plain x2, k_fct_limit, R+/R- halo, "
                     "k_fct_update, halos)", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                     "algorithmic_bytes_per_cell": TRACER_BYTES},
        "kernel_launches_per_tracer_step": launches / (k * c.QA),
        "min_tracer_after": qmin, "tracer_mass_change_rel": [(a - b) / b if b else 0.0 for a, b in zip(rq, rq0)],
        "sections_ms_per_large_step": {kk: v[1] / k for kk, v in prof.items()},
        "limiter_form": "fused (k_fct_limit, R+/R- halo, k_fct_update)",
        "three_kernel_limiter": three_kernel,
        "mixed": mixed,
    }


def run_mixed_large(args, hevi, torch):
    """The multi-bubble configuration at its full 1024x1024x96 size: the same
    short steps (numfilter + RK4 + boundary/halo) from the same initial state
    in FP64 and in mixed precision, timed on the library stream over
    args.mixed_large_steps steps after the warm-up; both paths then run on,
    untimed, to args.mixed_error_steps steps in all, after which the errors of
    the mixed state against the FP64 state are taken, relative to each field's
    largest magnitude over the interior, with the FP64 mass and energy totals
    of both states."""
    from scale_b200 import mkinit

    w0 = time.time()
    c = mkinit.config(4, scale=args.mixed_scale)
    RT2P, DPRES0, REF_rhot = mkinit.large_prep(c)
    prep_s = time.time() - w0
    g = c.g
    N3 = int(np.prod(g.shape))
    cells = g.cells
    hevi.setup(g.index_dict(), c.scheme, c.scheme_tracer)
    try:
        hevi.stage_autotune(True)
        st0 = torch.empty((5, N3), dtype=torch.float64, device="cuda")
        for v, n in enumerate(("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")):
            st0[v].copy_(to_dev(c.state[n], torch))
        ref = {n: to_dev(v, torch) for n, v in c.ref.items()}
        dp0, rt2p, refr = to_dev(DPRES0, torch), to_dev(RT2P, torch), to_dev(REF_rhot, torch)
        del RT2P, DPRES0, REF_rhot
        GS = torch.ones(7 * N3, dtype=torch.float64, device="cuda")
        J0 = torch.zeros(7 * N3, dtype=torch.float64, device="cuda")
        MAPF = torch.ones(g.IA * g.JA * 8, dtype=torch.float64, device="cuda")
        cor = torch.zeros(g.IA * g.JA, dtype=torch.float64, device="cuda")
        wd = np.zeros(g.KA)
        grid = dict(CDZ=g.CDZ, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY,
                    RFDZ=g.RFDZ, RFDX=g.RFDX, RFDY=g.RFDY)
        stream = torch.cuda.ExternalStream(hevi.stream_handle())
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k, warm = args.mixed_large_steps, max(3, args.warmup)
        total = max(warm + k, args.mixed_error_steps)

        def run(mixed):
            ft = torch.float32 if mixed else torch.float64
            st = st0.clone()
            X = dict(DENS=st[0], MOMZ=st[1], MOMX=st[2], MOMY=st[3], RHOT=st[4])
            z = lambda q=1: torch.zeros(q * N3, dtype=ft, device="cuda")  # noqa: E731
            mflx, tflx, nd = z(3), z(3), z(15)
            tend = {n: z() for n in ("DENS_t", "MOMZ_t", "MOMX_t", "MOMY_t", "RHOT_t")}
            nf = hevi.ATMOS_DYN_numfilter_coef_mixed_dev if mixed else hevi.ATMOS_DYN_numfilter_coef_dev
            rk = hevi.ATMOS_DYN_Tinteg_short_rk4_mixed_dev if mixed else hevi.ATMOS_DYN_Tinteg_short_rk4_dev

            def step():
                nf(num_diff=nd, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, DT=c.dt,
                   REF_dens=ref["REF_dens"], REF_pott=ref["REF_pott"], ND_COEF=c.nd_coef, ND_ORDER=1,
                   ND_SFC_FACT=1.0, ND_USE_RS=True, **X)
                rk(PROG=None, mflx_hi=mflx, tflx_hi=tflx, DPRES0=dp0, RT2P=rt2p, CORIOLI=cor, num_diff=nd,
                   wdamp_coef=wd, divdmp_coef=0.0, DDIV=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False,
                   FLAG_FCT_ALONG_STREAM=True, PHI=ref["PHI"], GSQRT=GS, J13G=J0, J23G=J0, J33G=1.0, MAPF=MAPF,
                   REF_dens=ref["REF_dens"], REF_rhot=refr, BND_W=False, BND_E=False, BND_S=False, BND_N=False,
                   dt=c.dt, **X, **tend, **grid)
                hevi.boundary_dev(**X)

            for _ in range(warm):
                step()
            hevi.check()
            torch.cuda.synchronize()
            hevi.profile(True)
            t0.record(stream)
            for _ in range(k):
                step()
            t1.record(stream)
            torch.cuda.synchronize()
            prof = hevi.profile_report()
            hevi.profile(False)
            hevi.check()
            ms = t0.elapsed_time(t1) / k
            for _ in range(total - warm - k):  # on to the step of the error comparison, untimed
                step()
            hevi.check()
            torch.cuda.synchronize()
            mass = hevi.domain_sum_dev(X["DENS"], g.CDZ, g.CDX, g.CDY)
            eng = hevi.energy_sum_dev(**X, CZ=g.CZ, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY)
            del mflx, tflx, nd, tend
            return st, ms, prof, mass, eng

        X0 = dict(DENS=st0[0], MOMZ=st0[1], MOMX=st0[2], MOMY=st0[3], RHOT=st0[4])
        mass0 = hevi.domain_sum_dev(X0["DENS"], g.CDZ, g.CDX, g.CDY)
        eng0 = hevi.energy_sum_dev(**X0, CZ=g.CZ, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY)
        st64, ms64, prof64, mass64, eng64 = run(False)
        st32, ms32, prof32, mass32, eng32 = run(True)
        sl = (slice(g.KS - 1, g.KE), slice(g.IS - 1, g.IE), slice(g.JS - 1, g.JE))
        errs = {}
        for v, n in enumerate(("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")):
            a64 = st64[v].view(g.JA, g.IA, g.KA).permute(2, 1, 0)[sl[0], sl[1], sl[2]]
            a32 = st32[v].view(g.JA, g.IA, g.KA).permute(2, 1, 0)[sl[0], sl[1], sl[2]]
            d = (a32 - a64).abs()
            scale = float(a64.abs().max())
            errs[n] = {"max": float(d.max()) / scale, "rms": float(d.pow(2).mean().sqrt()) / scale}
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        n64, t64 = prof64.get("hevi_stage", (0, 0.0))
        n32, t32 = prof32.get("hevi_stage_mixed", (0, 0.0))
        s64, s32 = t64 / max(n64, 1), t32 / max(n32, 1)

        def leg_roofline(stage_bytes, step_bytes, stage_ms, step_ms, r):
            ach = stage_bytes * cells / (stage_ms * 1e-3) / 1e9 if stage_ms else None
            return {"bound": "hbm", "kernel": stage_form_name(hevi, r), "achieved": ach, "peak": hbm,
                    "peak_source": "measured" if "hbm_gbs" in peaks else "fallback", "unit": "GB/s",
                    "frac": ach / hbm if ach else None, "algorithmic_bytes_per_launch": stage_bytes * cells,
                    "algorithmic_bytes_per_cell": stage_bytes, "stage_ms": stage_ms,
                    "step_frac": step_bytes * cells / (step_ms * 1e-3) / 1e9 / hbm}
        return {
            "workload": f"{g.IMAX}x{g.JMAX}x{g.KMAX} multi-bubble (32 seeded bubbles +1..3 K), dx=dz=200 m, UD3, dt=0.4 s",
            "cells": cells, "steps": k, "input_prep_s": prep_s,
            "fp64": {"value": cells / (ms64 * 1e-3), "ms_per_step": ms64, "stage_ms": s64,
                     "stage_frac_of_measured_hbm": STAGE_BYTES * cells / (s64 * 1e-3) / 1e9 / hbm if s64 else None,
                     "roofline": leg_roofline(STAGE_BYTES, STEP_BYTES, s64, ms64, "double"),
                     "sections_ms_per_step": {q: v[1] / k for q, v in prof64.items()}},
            "mixed": {"value": cells / (ms32 * 1e-3), "ms_per_step": ms32, "stage_ms": s32,
                      "stage_frac_of_measured_hbm": MIXED_STAGE_BYTES * cells / (s32 * 1e-3) / 1e9 / hbm if s32 else None,
                      "step_frac_of_measured_hbm": (4 * MIXED_STAGE_BYTES + MIXED_NUMFILTER_BYTES) * cells
                      / (ms32 * 1e-3) / 1e9 / hbm,
                      "roofline": leg_roofline(MIXED_STAGE_BYTES, 4 * MIXED_STAGE_BYTES + MIXED_NUMFILTER_BYTES, s32,
                                               ms32, "float"),
                      "sections_ms_per_step": {q: v[1] / k for q, v in prof32.items()}},
            "speedup_mixed_vs_fp64": ms64 / ms32,
            "error_vs_fp64": {"steps": total, "fields": errs,
                              "max_over_fields": max(e["max"] for e in errs.values()), "target": 1e-5},
            "budgets_after_error_steps": {
                "mass_drift_rel": {"fp64": (mass64 - mass0) / mass0, "mixed": (mass32 - mass0) / mass0},
                "ENGT_change_rel": {"fp64": (eng64["ENGT"] - eng0["ENGT"]) / eng0["ENGT"],
                                    "mixed": (eng32["ENGT"] - eng0["ENGT"]) / eng0["ENGT"]},
                "ENGT_mixed_vs_fp64_rel": (eng32["ENGT"] - eng64["ENGT"]) / eng64["ENGT"]},
            "autotune": hevi.autotune_report(),
        }
    finally:
        hevi.finalize()


def run_ensemble(args, hevi, torch):
    """The 48-member uneven ensemble (16 each of 64x64x64, 128x128x96 and
    256x256x96), advanced two ways on the same inputs: every kernel of a short
    step launched once over all members with the step replayed as a CUDA graph
    and the stage shape autotuned, and the whole short step as ONE persistent
    cooperative launch (also replayed as a graph)."""
    from scale_b200 import mkinit
    from scale_b200.ensemble import Ensemble

    w0 = time.time()
    cases = mkinit.ensemble(scale=args.ensemble_scale)
    prep_s = time.time() - w0
    cells = sum(c.g.cells for c in cases)
    sizes = {}
    for c in cases:
        k = f"{c.g.IMAX}x{c.g.JMAX}x{c.g.KMAX}"
        sizes[k] = sizes.get(k, 0) + 1
    k = args.ensemble_steps

    def timed(e):
        e.capture(1)  # one eager step (tunes the stage shape / builds the block maps), then one recorded step
        e.run(max(3, args.warmup))
        hevi.check()
        stream = torch.cuda.ExternalStream(hevi.stream_handle())
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        l0 = hevi.kernel_launches()
        t0.record(stream)
        e.run(k)
        t1.record(stream)
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1)
        launches = hevi.kernel_launches() - l0
        hevi.check()
        return ms, launches

    e = Ensemble(cases)
    try:
        hevi.stage_autotune(True)
        ms, launches = timed(e)
        shape = hevi.stage_shape_get()
        out = {"value": cells * k / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / k, "steps": k,
               "members": len(e.shapes), "sizes": sizes, "cells": cells,
               "kernel_launches_per_step": launches / k, "cuda_graph": True,
               "stage_shape": {"tile_x": shape[0], "raster": shape[1]}, "autotune": hevi.autotune_report(),
               "input_prep_s": prep_s, "l2": "inputs larger than L2"}
    finally:
        e.close()
    e = Ensemble(cases, persistent=True)
    del cases
    try:
        ms, launches = timed(e)
        out["persistent"] = {
            "value": cells * k / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / k, "steps": k,
            "kernel_launches_per_step": launches / k, "ctas": hevi.persistent_grid(), "cuda_graph": True,
            "step": "numerical filter + RK4 of 4 HEVI stages + boundary values and halos as one cooperative launch "
                    "(scale_hevi_short_step_persistent_dev), fused stage form, tile width 16",
        }
    finally:
        e.close()
    return out


def run_adjoint(args, hevi, torch):
    """Gradient of the warm-bubble cost (128x128x64, UD3): J = 1/2 sum of
    (theta - theta_base)^2 vol over x, y in [20, 44] km, z in [2, 6] km after
    120 short steps, with respect to the initial theta, MOMX and MOMY, by the
    adjoint with a checkpoint every 10 steps; checked against central finite
    differences (eps = 1e-6) along 8 seeded directions and by the
    tangent-linear dot-product test. The differentiated window starts after
    10 short steps of spin-up from rest (at rest every face velocity is
    exactly zero, where the UD3 upwind switches have no derivative)."""
    from scale_b200 import adjoint, mkinit

    out = {}
    for scheme in ("UD3", "CD4"):
        c = mkinit.config(5)
        c.scheme = scheme
        hevi.setup(c.g.index_dict(), c.scheme, c.scheme_tracer)
        try:
            p = adjoint.Problem(c, nsteps=args.adjoint_steps, K=10, spinup=10)
            torch.cuda.synchronize()
            w0 = time.time()
            J, _ = p.value_and_grad()
            torch.cuda.synchronize()
            t_grad = time.time() - w0
            X = p.model.state()
            p.model.boundary(X)
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            lam = torch.ones_like(X)
            p.model.adjoint(X, lam)  # warm
            t0.record()
            for _ in range(5):
                p.model.adjoint(X, lam)
            t1.record()
            torch.cuda.synchronize()
            ms_adj = t0.elapsed_time(t1) / 5
            t0.record()
            for _ in range(5):
                p.model.step(X)
            t1.record()
            torch.cuda.synchronize()
            ms_fwd = t0.elapsed_time(t1) / 5
            hevi.check()
            eps_list = (1e-6, 1e-5, 1e-4)
            r = adjoint.gradient_check(p, ndirs=8, eps=eps_list)
            X = p.model.state()
            p.model.boundary(X)
            dp = adjoint.dot_product_test(p.model, X, 3)
            fd = {}
            for e in eps_list:
                errs = sorted(d[f"rel_err_{e:g}"] for d in r["directions"])
                fd[f"{e:g}"] = {"max": errs[-1], "median": errs[len(errs) // 2]}
            out[scheme] = {"J": J, "gradient_s": t_grad, "steps": args.adjoint_steps, "checkpoint_every": 10,
                           "ms_per_adjoint_step": ms_adj, "ms_per_forward_step": ms_fwd,
                           "adjoint_cost_vs_forward": ms_adj / ms_fwd,
                           "fd_rel_err_by_eps": fd, "directions": len(r["directions"]),
                           "dot_product_rel_diff": dp["rel_diff"]}
            # the same directions with both perturbed runs in double-double
            # arithmetic (scale_hevi_short_step_dd_dev), at the configuration's eps
            w0 = time.time()
            rdd = adjoint.gradient_check(p, ndirs=8, eps=1e-6, dd=True)
            errs = sorted(d["rel_err"] for d in rdd["directions"])
            out[scheme]["fd_rel_err_double_double"] = {
                "eps": 1e-6, "max": errs[-1], "median": errs[len(errs) // 2], "seconds": time.time() - w0,
                "forward": "pass-form short step in double-double arithmetic (about 32 digits)"}
        finally:
            hevi.finalize()
    out["workload"] = "warm bubble 128x128x64, dx=500 m, dt=1 s; J over x,y in [20,44] km, z in [2,6] km"
    return out


def stage_form_name(hevi, r="double"):
    """The kernels of one HEVI stage in the stage form the library runs now."""
    tx, raster = hevi.stage_shape_get(r == "float")
    if tx == 0:
        return f"one HEVI stage: k_hevi_explicit<{r}> + k_hevi_column<{r}> (tiled form)"
    return f"one HEVI stage: k_hevi_stage<{r}> (fused form, tile width {tx}, raster {raster})"


def read_traffic():
    """DRAM bytes per HEVI stage from the committed ncu summary, if present."""
    p = ROOT / "profiles" / "hevi_stage_512x512x128.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_stage_full_size:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def run_e2e(args, c, hevi, torch):
    """Large steps through the host-array plugin entry (ATMOS_DYN_Tstep_large_fvm_heve),
    pinned host buffers, copies inside the timed region."""
    from scale_b200 import mkinit

    g = c.g

    def pinned(a):
        t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
        v = t.numpy()
        v[:] = np.ravel(a, order="K")
        return t, v.reshape(a.shape, order="F")

    keep = []

    def P(a):
        t, v = pinned(a)
        keep.append(t)
        return v

    st = {n: P(c.state[n]) for n in ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")}
    q = P(c.state["QTRC"])
    tp = {n: P(g.zeros()) for n in ("DENS_tp", "MOMZ_tp", "MOMX_tp", "MOMY_tp", "RHOT_tp")}
    rq = P(g.zeros(c.QA))
    mf, tf, nd = P(g.zeros(3)), P(g.zeros(3)), P(g.zeros(5, 3))
    ref = {n: P(v) for n, v in c.ref.items()}
    cor = P(np.zeros((g.IA, g.JA), order="F"))
    GS = np.ones(g.shape + (7,), order="F")
    J0 = np.zeros(g.shape + (7,), order="F")
    MAPF = np.ones((g.IA, g.JA, 2, 4), order="F")
    R, CV, CP, M = mkinit.aq_props(c.QA)
    nstep = int(np.ceil((c.dtl - mkinit.EPS) / c.dt))

    def call():
        hevi.ATMOS_DYN_Tstep_large_fvm_heve(
            QTRC=q, QA=c.QA, mflx_hi=mf, tflx_hi=tf, num_diff=nd, RHOQ_tp=rq, CORIOLI=cor, CDZ=g.CDZ, CDX=g.CDX,
            CDY=g.CDY, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY, RFDZ=g.RFDZ,
            RFDX=g.RFDX, RFDY=g.RFDY, PHI=ref["PHI"], GSQRT=GS, J13G=J0, J23G=J0, J33G=1.0, MAPF=MAPF, AQ_R=R,
            AQ_CV=CV, AQ_CP=CP, AQ_MASS=M, REF_dens=ref["REF_dens"], REF_pott=ref["REF_pott"],
            REF_pres=ref["REF_pres"], ND_COEF=c.nd_coef, ND_ORDER=1, ND_SFC_FACT=1.0, ND_USE_RS=True,
            wdamp_coef=np.zeros(g.KA), divdmp_coef=0.0, FLAG_FCT_TRACER=c.fct, FLAG_FCT_ALONG_STREAM=True,
            DTLS=c.dtl, DTSS=c.dt, **st, **tp)

    call()  # warm-up (first call also checks the metric arrays once)
    stream = torch.cuda.ExternalStream(hevi.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ncall = args.e2e_calls
    torch.cuda.synchronize()
    b0 = hevi.transfer_bytes()
    e0.record(stream)
    for _ in range(ncall):
        call()
    e1.record(stream)
    torch.cuda.synchronize()
    b1 = hevi.transfer_bytes()
    ms = e0.elapsed_time(e1) / ncall
    h2d = (b1[0] - b0[0]) // ncall
    d2h = (b1[1] - b0[1]) // ncall
    return {"value": g.cells * nstep / (ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "ms_per_step": ms, "step": f"one large step through the host-array entry ATMOS_DYN_Tstep_large_fvm_heve_b200 "
                                      f"({nstep} short steps + RK3 advection of {c.QA} tracers with FCT), pinned host buffers",
            "calls": ncall}


# ---------------------------------------------------------------------------
# CPU timings of the oracle (restatement of the reference's FP64 CPU code)
# ---------------------------------------------------------------------------
def oracle_short_step_rate(scale: float, steps: int, min_seconds: float = 0.0, max_steps: int = 100):
    import oracle
    from scale_b200 import mkinit

    c, RT2P, DPRES0, REF_rhot = make_inputs(scale)
    g = c.g
    GS, J13, J23, MAPF = oracle.flat_metrics(g)
    nd = g.zeros(5, 3)
    x = {n: c.state[n] for n in ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")}
    x["mflx_hi"], x["tflx_hi"] = g.zeros(3), g.zeros(3)
    a = dict(DENS_t=g.zeros(), MOMZ_t=g.zeros(), MOMX_t=g.zeros(), MOMY_t=g.zeros(), RHOT_t=g.zeros(),
             DPRES0=DPRES0, RT2P=RT2P, CORIOLI=np.zeros((g.IA, g.JA), order="F"), num_diff=nd,
             wdamp_coef=np.zeros(g.KA), divdmp_coef=0.0, DDIV=g.zeros(), CDZ=g.CDZ, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY,
             RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY, RFDZ=g.RFDZ, RFDX=g.RFDX, RFDY=g.RFDY, PHI=c.ref["PHI"],
             GSQRT=GS, J13G=J13, J23G=J23, J33G=1.0, MAPF=MAPF, REF_dens=c.ref["REF_dens"], REF_rhot=REF_rhot,
             dt=c.dt)
    times = []
    while len(times) < steps or (sum(times) < min_seconds and len(times) < max_steps):
        t = time.perf_counter()
        oracle.numfilter(g, nd, x, c.ref, DT=c.dt, ND_COEF=c.nd_coef)
        oracle.tinteg_short_rk4(g, c.scheme, x, a)
        for n in ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT"):
            oracle.halo(g, x[n])
        times.append(time.perf_counter() - t)
    return g, times, oracle.num_threads()


def cpu_baseline(args):
    g, times, threads = oracle_short_step_rate(args.cpu_scale, 2, min_seconds=args.cpu_seconds)
    rate = g.cells / statistics.median(times)
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(times)} short steps (numfilter + RK4 + halo) of the same configuration on a "
                      f"{g.IMAX}x{g.JMAX}x{g.KMAX} horizontal sub-domain, FP64 C restatement with OpenMP; "
                      f"median {statistics.median(times):.2f} s per step"}


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return
    g, times, threads = oracle_short_step_rate(args.cpu_scale, args.steps + args.warmup)
    t = times[args.warmup:] or times
    rate = g.cells / statistics.median(t)
    out = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world, "steps": len(t),
           "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(t), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; no dataset involved)",
           "config": {"workload": f"512x512x128 CD4 short step sampled on a {g.IMAX}x{g.JMAX}x{g.KMAX} sub-domain",
                      "cells": g.cells},
           "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": f"short steps on a {g.IMAX}x{g.JMAX}x{g.KMAX} sub-domain of the same "
                                      "configuration: FP64 C restatement of the reference Fortran (no Fortran "
                                      "compiler in the image), OpenMP over all host threads"},
           "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--scale", type=float, default=1.0, help="horizontal scale of the workload (1 = 512x512)")
    ap.add_argument("--cpu-scale", type=float, default=0.25, help="horizontal scale of the CPU sample")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="minimum CPU work of the baseline sample")
    ap.add_argument("--e2e-calls", type=int, default=2)
    ap.add_argument("--stage-shape", default="", help="fixed stage form 'tile_x,raster' (0 = tiled) instead of the autotuner")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision measurement")
    ap.add_argument("--no-heve", action="store_true", help="skip the HEVE short-step measurement")
    ap.add_argument("--no-tracer", action="store_true", help="skip the tracer advection measurement")
    ap.add_argument("--tracer-steps", type=int, default=10, help="timed large steps of the tracer leg")
    ap.add_argument("--no-terrain", action="store_true", help="skip the terrain-following short-step measurement")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 48-member ensemble measurement")
    ap.add_argument("--ensemble-steps", type=int, default=20)
    ap.add_argument("--ensemble-scale", type=float, default=1.0, help="horizontal scale of the ensemble members")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint gradient measurement")
    ap.add_argument("--no-mixed-large", action="store_true", help="skip FP64 vs mixed on 1024x1024x96")
    ap.add_argument("--mixed-large-steps", type=int, default=20)
    ap.add_argument("--mixed-error-steps", type=int, default=600, help="steps before the mixed-vs-FP64 error is taken")
    ap.add_argument("--mixed-scale", type=float, default=1.0, help="horizontal scale of the 1024x1024x96 leg")
    ap.add_argument("--adjoint-steps", type=int, default=120)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        log("warm-up raised to the minimum of 3 steps")
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
