#!/usr/bin/env python
"""Benchmark of the B200 Lagrangian DG time step (Lag2D curved-P2 path).

Metric: DOF-updates/s per RK stage, FP64 = N_cells * ndegr * nq * stages / time.
Workload: Taylor-Green vortex on [0,1]^2, 1024 x 1024 curved-capable 9-node
quads (1,048,576 cells, 4,198,401 nodes), P2 Taylor basis, gamma 5/3, RK3,
Persson + WENO limiting, energy source on; synthetic initial state, no input
files.  A "step" is one full time step (3 RK stages) on the device-resident
state, replayed from a CUDA graph.

Usage:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
For N > 1 launch under torch.distributed.run; every rank runs an independent
replica (the path does not shard), timings are device events, max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DOF-updates/s per RK stage, FP64 vs FP32-mixed; adjoint/forward time ratio"
UNIT = "DOF-updates/s"
WORKLOAD = "tgv1024"
CPU_SAMPLE = "tgv64"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dtfix", type=float, default=0.0,
                    help="fixed time step (ndt = 0) instead of the CFL one, for the configurations whose "
                         "CFL steps break the scheme (Noh, hybrid Sedov)")
    ap.add_argument("--rho0", action="store_true", help="per-cell initial densities 1 + 0.01 N(0, 1)")
    ap.add_argument("--no-p1", action="store_true", help="skip the linear P1 (Sod) block")
    ap.add_argument("--adjoint-steps", type=int, default=4)
    ap.add_argument("--adjoint-checkpoint", type=int, default=2)
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def host_info():
    """CPU model (as lscpu reports it, from /proc/cpuinfo) and the number of
    host threads the process may use."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    return {"cpu_model": model, "nproc": n}


def config_block(name, mesh, cfg, n):
    out = {"workload": name, "cells": mesh.ncell, "triangles": mesh.ntria, "nodes": mesh.npoin,
           "basis": "P2 Taylor (ndegr=6, nq=4)", "rk_stages": cfg.nstag, "limiter": "Persson + WENO",
           "gamma": cfg.gamlg, "cfl": cfg.cfl, "parallelism": f"replicas x{n}",
           "l2": ("working set > 126 MB L2 (no flush needed)" if mesh.ncell >= 262144
                  else "working set within the 126 MB L2 (small configuration)")}
    if cfg.ndt == 0:
        out["dt"] = f"fixed {cfg.dtfix:g}"
    out["host"] = host_info()
    return out


def make_case(args):
    """The workload of --workload, with the --dtfix and --rho0 options applied."""
    import dataclasses
    from lag2d_b200.config import initial_density_factors, workload
    m, c = workload(args.workload)
    if args.dtfix > 0:
        c = dataclasses.replace(c, ndt=0, dtfix=args.dtfix)
    rho0 = initial_density_factors(m) if args.rho0 else None
    return m, c, rho0


def new_solver(m, c, rho0, **kw):
    from lag2d_b200.api import Lag2DSolver
    s = Lag2DSolver(m, c, **kw)
    if rho0 is not None:
        s.set_rho0(rho0)
    s.init_fields()
    return s


# --------------------------------------------------------------------------
# CPU baseline: the oracle (C restatement of the reference), single thread
# --------------------------------------------------------------------------
def _cpu_worker(args):
    name, warm, nsteps = args
    sys.path.insert(0, ROOT)
    import numpy as np
    from lag2d_b200.config import workload
    from oracle.oracle import Oracle
    m, c = workload(name)
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    coord = m.coord.copy()
    ustar = np.zeros_like(coord)
    dt, ta = c.dtfix, 0.0
    it = 1
    if warm:
        _, dt, ta = o.run(unkno, coord, m.coord, geoel, amatr, ustar, it, warm, dt, ta)
        it += warm
    times = []
    for _ in range(nsteps):
        t0 = time.perf_counter()
        _, dt, ta = o.run(unkno, coord, m.coord, geoel, amatr, ustar, it, 1, dt, ta)
        times.append(time.perf_counter() - t0)
        it += 1
    return m.ncell, c.nstag, times


def cpu_baseline(seconds: float):
    """Time the oracle on a bounded sample of the workload (single thread)."""
    ncell, nstag, t = _cpu_worker((CPU_SAMPLE, 0, 1))
    per_step = max(t[0], 1e-3)
    nsteps = max(2, int(seconds / per_step))
    ncell, nstag, times = _cpu_worker((CPU_SAMPLE, 0, nsteps))
    total = sum(times)
    value = ncell * 24 * nstag * nsteps / total
    return {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{CPU_SAMPLE}: Taylor-Green 64x64 P2 quads (same step: Persson+WENO, RK3), "
                      f"{nsteps} steps, {total:.1f} s, oracle C restatement -O2 single thread",
            "host": host_info()}


def run_reference(args):
    rank, local_rank, world = dist_env()
    if rank != 0:
        return 0
    import multiprocessing as mp
    from lag2d_b200.config import workload
    m, c = workload(args.workload)
    nproc = host_info()["nproc"]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(nproc) as pool:
        res = pool.map(_cpu_worker, [(CPU_SAMPLE, args.warmup, args.steps)] * nproc)
    wall = time.perf_counter() - t0
    ncell, nstag = res[0][0], res[0][1]
    per_step_max = [max(ts) for ts in zip(*[r[2] for r in res])]
    elapsed = sum(per_step_max)
    value = nproc * ncell * 24 * nstag * args.steps / elapsed
    sample = (f"{CPU_SAMPLE}: Taylor-Green 64x64 P2 quads per process, {nproc} processes x {args.steps} timed "
              f"steps (after {args.warmup} warm-up), oracle C restatement of the reference step "
              f"(the Fortran reference cannot be compiled here), wall {wall:.1f} s")
    cfgb = config_block(args.workload, m, c, args.gpus)
    # the metric is per-cell work, so the 1024^2 rate is sampled on independent
    # 64^2 problems, one per host thread (a whole 1024^2 step takes ~55 s on one thread)
    cfgb["cpu_sample"] = (f"{CPU_SAMPLE} (64x64 P2 quads, same step) x {nproc} independent processes, "
                          f"DOF-updates/s summed over processes")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": cfgb,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(index)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = sorted(float(r[1]) for r in rows if len(r) > 8 and r[1].strip().replace(".", "").isdigit())
        mx = [float(r[2]) for r in rows if len(r) > 8 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows if len(r) > 8 for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def fp64_peak():
    """Measured FP64 FMA throughput of this GPU (TFLOP/s, best of 3 launches of
    independent FMA chains on every SM, CUDA events); None if the measurement
    library is missing."""
    import ctypes
    lib_path = os.path.join(ROOT, "lag2d_b200", "_lib", "liblag2d_bench.so")
    if not os.path.exists(lib_path):
        return None
    lib = ctypes.CDLL(lib_path)
    lib.lag2d_bench_dfma_tflops.restype = ctypes.c_double
    lib.lag2d_bench_dfma_tflops.argtypes = [ctypes.c_int, ctypes.c_int]
    tf = lib.lag2d_bench_dfma_tflops(200000, 3)
    return tf if tf > 0 else None


def measured_flops(family, ncell):
    """FP64 FLOPs per launch of a kernel family (2 per DFMA, 1 per DMUL/DADD,
    from ncu's executed-instruction counters of a capture, per cell in
    profiles/flops.json), scaled to this workload's cells; None when no
    capture is recorded."""
    try:
        with open(os.path.join(ROOT, "profiles", "flops.json")) as f:
            t = json.load(f)
        return t[family]["fp64_flops_per_cell"] * ncell
    except Exception:
        return None


def measured_traffic(family, ncell):
    """DRAM bytes per launch of a kernel family from the committed ncu summary
    (profiles/traffic.json: bytes per cell of a capture larger than L2),
    scaled to this workload's cells; None when no capture is recorded."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
        return t[family]["dram_bytes_per_cell"] * ncell
    except Exception:
        return None


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def adjoint_block(s, args, fwd_ms_per_step, state, grads=None):
    """Time lag2d_adjoint over a short window starting from ``state`` (unkno,
    coord, ustar, itime, dtfix, tacru): the reverse sweep per step (excluding
    the segment recompute) over the forward step time of the main timing; the
    recompute is reported beside it.  The gradients are returned in
    ``grads`` (a dict) when given."""
    import numpy as np
    from lag2d_b200.api import Lag2DError

    nsteps, k = args.adjoint_steps, args.adjoint_checkpoint
    if nsteps <= 0:
        return {"ratio": None, "note": "not run (--adjoint-steps 0)"}
    u0, x0, us0, it0, dt0, ta0 = state
    try:
        for K in (1, k):                      # the first call loads the reverse kernels
            s.set_state(u0, x0, us0)
            s.itime, s.dtfix, s.tacru = it0, dt0, ta0
            J, gu, gx, gs, ms = s.adjoint(nsteps, K)
    except Lag2DError as e:
        return {"ratio": None, "note": str(e)}
    if grads is not None:
        grads.update(J=J, gu=gu, gx=gx, gs=gs)
    rev = ms[2] / nsteps
    return {"ratio": rev / fwd_ms_per_step, "reverse_ms_per_step": rev,
            "recompute_ms_per_step": ms[1] / nsteps, "forward_with_checkpoints_ms_per_step": ms[0] / nsteps,
            "forward_ms_per_step": fwd_ms_per_step, "steps": nsteps, "checkpoint_every": k,
            "functional": "J = 1/2 sum_c m_c (u_c^2 + v_c^2) at the window end",
            "grad_finite": bool(np.isfinite(gu).all() and np.isfinite(gx).all()),
            "precision": ("FP32-mixed (volume-integral and sub-cell-mass transposes in FP32)"
                          if s._c.precision == 1 else "FP64")}


def p1_block(args, timed, families):
    """Throughput of the linear P1 path on the Sod workloads (DOF-updates/s
    per RK stage, 12 DOFs per cell), its kernel split and stage roofline, and
    the oracle timed on the reference's 200 x 10 case."""
    from lag2d_b200.config import workload
    from lag2d_b200.roofline import stage_bytes_p1
    peak, peak_kind = peaks()
    names = ("bounds", "cell", "node", "rhs", "dt", "update", "nodes", "geom", "copy")
    out = {"path": "ncurv=0, nfint=1, nlimi=6 (linear P1, straight quads); parity: bit for bit with the "
                   "oracle in the no-FMA build (tests/test_gpu_p1.py, tests/test_gpu_rz.py)",
           "noh_rz100_note": "Noh implosion in RZ (nrz=1, y the radius): the spherical implosion on 100x100 quads",
           "noh_rzaw100_note": "the same in the area-weighted RZ form (nrz=2): per-stage mass centre and mass "
                               "matrix, geometry after every stage"}
    for name in ("sod200", "sod1024", "noh_rz100", "noh_rzaw100"):
        m, c = workload(name)
        s = new_solver(m, c, None)
        ms, done, launches = timed(s)
        dof_stage = m.ncell * c.ndegr * c.nq
        ms_step = ms / max(done, 1)
        fams = families(s, names)
        sb = stage_bytes_p1(m.ncell, m.npoin)
        gbs = sb / (ms_step / c.nstag / 1e3) / 1e9
        out[name] = {"value": dof_stage * c.nstag * done / (ms / 1e3), "unit": UNIT, "ms_per_step": ms_step,
                     "steps": done, "cells": m.ncell, "nodes": m.npoin, "rk_stages": c.nstag,
                     "gpu_launches": launches,
                     "kernels_ms_per_step": {f: v["ms_per_launch"] * v["launches"] / 2 for f, v in fams.items()},
                     "stage_roofline": {"bytes_per_stage": sb, "achieved_gbs": gbs, "peak": peak,
                                        "peak_kind": peak_kind, "frac": gbs / peak}}
        s.close()
    if not args.no_cpu_baseline:
        nc, nstag, times = _cpu_worker(("sod200", 0, 60))
        total = sum(times)
        out["sod200"]["cpu_baseline"] = {
            "value": nc * 12 * nstag * len(times) / total, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"sod200: the first {len(times)} steps, {total:.2f} s, oracle C restatement -O2 single thread"}
    return out


def run_ours(args):
    rank, local_rank, world = dist_env()
    import numpy as np
    import torch
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from lag2d_b200.replicas import aggregate_rate, max_over_ranks
    from lag2d_b200.roofline import kernel_bytes, stage_bytes

    m, c, rho0 = make_case(args)
    s = new_solver(m, c, rho0)
    sm = new_solver(m, c, rho0, precision=1)   # FP32-mixed form of the same step
    dof_stage = m.ncell * c.ndegr * c.nq

    def timed(solver):
        """K graph-replayed steps after W warm-up steps: device ms, steps, launches."""
        stream = torch.cuda.ExternalStream(solver.stream_ptr)
        solver.run(args.warmup)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = solver.kernel_launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        n = solver.run(args.steps)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1)), n, solver.kernel_launches - l0

    def families(solver, names=("persson", "weno", "src", "corner", "node", "rhs", "dt", "nodes", "geom", "copy")):
        solver.timing(True)
        solver.run(2)
        out = {}
        for f in names:
            k_ms, n = solver.kernel_ms(f)
            if k_ms is not None:
                out[f] = {"ms_per_launch": k_ms, "launches": n}
        solver.timing(False)
        return out

    # ---- timed regions (FP64, then FP32-mixed), clocks sampled across both
    clk = Clocks(local_rank)
    ms, done, launches = timed(s)
    ms_mx, done_mx, launches_mx = timed(sm)
    clocks = clk.stop()
    ms_per_step = ms / max(done, 1)
    value = aggregate_rate(dof_stage * c.nstag * done, ms / 1e3, world)
    value_mx = aggregate_rate(dof_stage * c.nstag * done_mx, ms_mx / 1e3, world)

    # ---- per-kernel device times (separate pass, events around each family)
    fams = families(s)
    fams_mx = families(sm)
    per_step = {f: v["ms_per_launch"] * v["launches"] / 2 for f, v in fams.items()}
    per_step_mx = {f: v["ms_per_launch"] * v["launches"] / 2 for f, v in fams_mx.items()}
    dom = max((f for f in per_step if f in ("src", "corner", "node", "rhs", "dt", "persson", "nodes", "geom")),
              key=lambda f: per_step[f])
    peak, peak_kind = peaks()
    kb = kernel_bytes(dom, m.ncell, m.npoin, c.nstag, source=c.ncase == 1)
    traffic = measured_traffic(dom, m.ncell)
    achieved = kb / (fams[dom]["ms_per_launch"] / 1e3) / 1e9
    sb = stage_bytes(m.ncell, m.npoin)
    stage_gbs = sb / (ms_per_step / c.nstag / 1e3) / 1e9

    # ---- error of the mixed form: both forms from the same initial state
    n_err = 10
    s.init_fields()
    sm.init_fields()
    s.run(n_err)
    sm.run(n_err)
    u64, x64 = s.get_state()[:2]
    umx, xmx = sm.get_state()[:2]
    nc = m.ncell
    diff = np.abs(umx[:nc, :, 0] - u64[:nc, :, 0])
    err_mx = np.minimum(diff / np.maximum(np.abs(u64[:nc, :, 0]), 1e-300),
                        diff / np.abs(u64[:nc, :, 0]).max(axis=0)).max(axis=0)
    mixed = {"value": value_mx, "unit": UNIT, "ms_per_step": ms_mx / max(done_mx, 1), "steps": done_mx,
             "speedup_vs_fp64": value_mx / value, "gpu_launches": launches_mx,
             "dtype": "f32 flux/quadrature arithmetic; f64 storage, nodal solve, nodes, volumes, cell averages",
             "cell_avg_err_vs_fp64": {"tau": float(err_mx[0]), "u": float(err_mx[1]), "v": float(err_mx[2]),
                                      "e": float(err_mx[3])},
             "node_err_vs_fp64": float(np.abs(xmx - x64).max()),
             "err_note": (f"max over cells after {n_err} steps from the same initial state, against the FP64 GPU "
                          "step (itself within 1e-12 of the FP64 oracle); relative to the value, or to the field "
                          "scale where the field crosses zero"),
             "kernels_ms_per_step": per_step_mx}
    sm.close()

    # ---- end to end through the C-ABI with pinned host buffers
    u_h = torch.empty((m.nsize, c.nq, c.ndegr), dtype=torch.float64, pin_memory=True)
    x_h = torch.empty((m.npoin, 2), dtype=torch.float64, pin_memory=True)
    us_h = torch.empty((m.npoin, 2), dtype=torch.float64, pin_memory=True)
    s.get_state_ptrs(u_h.data_ptr(), x_h.data_ptr(), us_h.data_ptr())
    h2d = 8 * (m.ncell * 24 + 4 * m.npoin)
    d2h = h2d
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        s.set_state_ptrs(u_h.data_ptr(), x_h.data_ptr(), us_h.data_ptr())
        s.step()
        s.get_state_ptrs(u_h.data_ptr(), x_h.data_ptr(), us_h.data_ptr())
    te = max_over_ranks(time.perf_counter() - t0)
    # the link these copies run on: one pinned copy of the same bytes each way,
    # CUDA events (a bound for the end-to-end step: step time + both copies)
    dev_buf = torch.empty(h2d // 8, dtype=torch.float64, device="cuda")
    host_buf = torch.empty(h2d // 8, dtype=torch.float64, pin_memory=True)
    link = {}
    for name, (dst, src) in (("h2d", (dev_buf, host_buf)), ("d2h", (host_buf, dev_buf))):
        best = None
        for _ in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            dst.copy_(src, non_blocking=True)
            b.record()
            b.synchronize()
            ms_c = a.elapsed_time(b)
            best = ms_c if best is None else min(best, ms_c)
        link[name] = {"ms": best, "gbs": h2d / (best / 1e3) / 1e9}
    del dev_buf, host_buf
    bound_ms = ms_per_step + link["h2d"]["ms"] + link["d2h"]["ms"]
    e2e = {"value": aggregate_rate(dof_stage * c.nstag * args.e2e_steps, te, world), "unit": UNIT,
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "ms_per_step": 1e3 * te / args.e2e_steps,
           "api": "lag2d_set_state + lag2d_step + lag2d_get_state (pinned host, Fortran layout)",
           "link": link,
           "bound": {"ms_per_step": bound_ms, "value": dof_stage * c.nstag / (bound_ms / 1e3),
                     "note": "device step + one pinned copy of the step's state each way (measured above)"}}

    # ---- adjoint: reverse sweep per step against the forward step time, FP64
    # and FP32-mixed from the same state (the FP64 solver's current one)
    u_a, x_a, us_a, _ = s.get_state()
    state = (u_a, x_a, us_a, s.itime, s.dtfix, s.tacru)
    g64, g32 = {}, {}
    adjoint = adjoint_block(s, args, ms_per_step, state, g64)
    sm2 = new_solver(m, c, rho0, precision=1)
    adjoint["fp32_mixed"] = adjoint_block(sm2, args, mixed["ms_per_step"], state, g32)
    sm2.close()
    if g64 and g32:
        import numpy as np
        rel = {}
        for key, name in (("gu", "dJ_dunkno"), ("gx", "dJ_dcoord"), ("gs", "dJ_dustar")):
            a, b = g32[key], g64[key]
            rel[name] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
        adjoint["fp32_mixed"]["grad_rel_l2_vs_fp64_adjoint"] = rel
        adjoint["fp32_mixed"]["J_rel_vs_fp64"] = abs(g32["J"] - g64["J"]) / abs(g64["J"])

    # ---- the linear P1 path (Sod on straight 4-node quads): the reference's
    # 200 x 10 configuration and a 1024 x 512 one, FP64, graph-replayed steps
    p1 = None if args.no_p1 else p1_block(args, timed, families)

    # ---- FP64 pipe: measured DFMA peak and each pass's FP64 FLOP rate
    tf_peak = fp64_peak() if rank == 0 else None
    fp64 = {"peak_tflops": tf_peak, "peak_kind": "measured (DFMA chains on every SM, CUDA events)",
            "per_kernel": {}}
    for f, v in fams.items():
        fl = measured_flops(f, m.ncell)
        if fl is None:
            continue
        tf = fl / (v["ms_per_launch"] / 1e3) / 1e12
        fp64["per_kernel"][f] = {"flops_per_launch": fl, "achieved_tflops": tf,
                                 "frac": (tf / tf_peak) if tf_peak else None}

    if rank == 0:
        # short summaries first: the line is long and readers may only see its head
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": done,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seedless structured mesh, analytic IC)",
                "config": config_block(args.workload, m, c, world), "clocks": clocks, "gpu_launches": launches,
                "e2e": e2e,
                "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                             "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                             "bytes_per_launch": kb},
                "fp32_mixed_summary": {"value": value_mx, "ms_per_step": mixed["ms_per_step"],
                                       "speedup_vs_fp64": mixed["speedup_vs_fp64"],
                                       "max_cell_avg_err_vs_fp64": max(mixed["cell_avg_err_vs_fp64"].values())},
                "adjoint_forward_ratio": adjoint.get("ratio"),
                "adjoint_forward_ratio_fp32_mixed": adjoint.get("fp32_mixed", {}).get("ratio")}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
        line.update({
            "stage_roofline": {"bytes_per_stage": sb, "achieved_gbs": stage_gbs, "peak": peak,
                               "frac": stage_gbs / peak, "roofline_dof_updates_per_s": dof_stage / (sb / (peak * 1e9))},
            "fp64_pipe": fp64, "kernels_ms_per_step": per_step, "fp32_mixed": mixed, "adjoint": adjoint})
        if p1 is not None:
            line["p1_sod"] = p1
        print(json.dumps(line), flush=True)
    s.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
