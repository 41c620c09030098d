#!/usr/bin/env python
"""Benchmark: 257^3 plasma-Poisson solves/s to 1e-10 relative residual.

Workload (the headline configuration): 257^3 cells on a 1 cm cube, relative
permittivity 1 in the gas and 4 in a 10-cell dielectric slab at z=0,
Dirichlet 0 V (z=0) and 1000 V (z=1), periodic x/y, right-hand side
e(n_i - n_e)/eps0 with lognormal densities (seeded synthetic stand-in).

One step = one complete solve from a zero initial guess to
||b - A x||_2 / ||b||_2 <= 1e-10, operator setup included, inputs resident in
HBM.  ``value`` is the mixed-precision solve (FP32 V-cycles inside FP64
refinement); the plain FP64 V-cycle solve is timed beside it (``fp64``).
``e2e`` repeats the mixed solve through the host C ABI (mps_linsolve) with
pinned host buffers, host<->device copies inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: one process per GPU (torchrun); the solve does not shard, every
rank solves its own replica (weak scaling), time = max over ranks.
--impl reference times the CPU restatement of the reference's own V-cycle
(perform_vcycle, oracle port) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))

import numpy as np  # noqa: E402

METRIC = "257³ Poisson solves/s @1e-10 rel. residual: mixed vs FP64 GPU; HBM GB/s"
UNIT = "solves/s"
N_DEFAULT = 257


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def workload_config(n, extra=None):
    cfg = {
        "workload": f"plasma Poisson {n}^3 cells, 1 cm cube, eps_r 1 / 4 (10-cell slab at z=0), "
                    f"Dirichlet 0 V / 1000 V on z, periodic x/y, e(n_i-n_e)/eps0 lognormal(ln 1e16, 1)",
        "cells": n ** 3,
        "tol_rel_residual": 1e-10,
        "hierarchy": "geom (l/2, odd cell merged, trilinear prolongation), RB-GS 2/2, coarsest <=125 cells dense",
        "initial_guess": "zero",
        "l2": "no flush: inputs (>=7 fields of 139 MB) exceed the 126 MB L2",
        "parallelism": "replicas",
    }
    if extra:
        cfg.update(extra)
    return cfg


from mps3d_b200.shard import barrier, dist_init, dist_max, gather_results, partition_by_cost  # noqa: E402


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, out_dir=None):
        self.gpu = gpu_index
        self.proc = None
        self.out_dir = out_dir
        self.path = None

    def __enter__(self):
        import tempfile

        try:
            if self.out_dir:
                os.makedirs(self.out_dir, exist_ok=True)
                self.path = os.path.join(self.out_dir, f"clocks_gpu{self.gpu}.csv")
            else:
                fd, self.path = tempfile.mkstemp(prefix=f"mps_clocks_gpu{self.gpu}_", suffix=".csv")
                os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not self.out_dir:
            try:
                os.remove(self.path)
            except OSError:
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
def host_cpu():
    """nproc, the CPU model (as lscpu names it) and the OpenMP threads used."""
    from oracle import oracle as orc

    return {"nproc": os.cpu_count(), "cpu_model": orc.cpu_model(), "threads": orc.get_threads(),
            "build": "gcc -O3 -march=native -fopenmp (built on this host)" if orc.native_loaded()
            else "gcc -O3 -march=x86-64-v2 -fopenmp"}


def oracle_cpu_solve(p, max_cycles=40, single_thread_cycles=1, tol=1e-10):
    """The FP64 restatement of perform_vcycle (the reference hierarchy,
    mgridlib/mgridsteps.f90:384-579) solving ``p`` from a zero guess: V-cycles
    on all host threads until the relative residual reaches ``tol`` (the
    reference's caller loop, poissoneq.f90:427-450, with the relative stop
    test), then ``single_thread_cycles`` more V-cycles on one thread.
    Returns per-cycle seconds (all threads), the residual history, the cycles
    the solve needed and the single-thread seconds per cycle."""
    from oracle import oracle as orc

    x = p.zeros_ghosted()
    b = orc.find_bvec(p)
    bn = np.linalg.norm(b)
    times, rel = [], []
    while len(rel) < max_cycles:
        t0 = time.perf_counter()
        rms = orc.vcycle(p, x)
        times.append(time.perf_counter() - t0)
        # the reference's RMS residual is sqrt(sum r^2 / N): relative L2 = rms*sqrt(N)/||b||
        rel.append(rms * np.sqrt(p.ncells) / bn)
        if rel[-1] <= tol:
            break
    need = len(rel) if rel[-1] <= tol else None
    t1 = None
    if single_thread_cycles:
        nthr = orc.get_threads()
        orc.set_threads(1)
        try:
            xs = x.copy()
            t0 = time.perf_counter()
            for _ in range(single_thread_cycles):
                orc.vcycle(p, xs)
            t1 = (time.perf_counter() - t0) / single_thread_cycles
        finally:
            orc.set_threads(nthr)
    return times, rel, need, t1


def reference_twin(n):
    """The reference's cell-centred hierarchy halves sizes by integer division
    (mgridsteps.f90:21-23) and drops the odd cell; on 2^k+1 sizes with periodic
    faces its V-cycle diverges, so the reference is timed on the power-of-two
    twin (same box, same physics, n-1 cells per direction)."""
    return n - 1 if n % 2 == 1 else n


def cpu_baseline_figures(n, problem=None, single_thread_cycles=1):
    """The reference's own V-cycle loop (oracle port, -march=native, OpenMP)
    solving the power-of-two twin of the workload to 1e-10 on the host cores:
    all-thread solves/s from the measured cycles, single-thread solves/s from
    ``single_thread_cycles`` cycles times the same cycle count."""
    from mps3d_b200 import workloads as W

    nt = reference_twin(n)
    p = problem if (problem is not None and nt == n) else W.plasma_poisson(nt)
    times, rel, need, t1 = oracle_cpu_solve(p, single_thread_cycles=single_thread_cycles)
    if need is None:
        raise RuntimeError(f"the oracle's V-cycle did not reach 1e-10 in {len(rel)} cycles: {rel[-3:]}")
    t_solve = float(sum(times))
    hc = host_cpu()
    out = {"value": 1.0 / t_solve, "unit": UNIT, "cores": hc["threads"], "kind": "port",
           "s_per_solve": t_solve, "vcycles": need, "s_per_cycle": t_solve / need,
           "single_thread": None if t1 is None else {"value": 1.0 / (t1 * need), "s_per_cycle": t1,
                                                     "cycles_timed": single_thread_cycles},
           "nproc": hc["nproc"], "cpu_model": hc["cpu_model"], "build": hc["build"],
           "rel_residual_history": rel,
           "sample": f"one full solve from zero to 1e-10 relative residual ({need} V-cycles, {t_solve:.1f} s) of the "
                     f"FP64 restatement of perform_vcycle on the {nt}^3 power-of-two twin of the {n}^3 problem "
                     f"(the reference hierarchy cannot coarsen {n}), {hc['threads']} OpenMP threads; single-thread: "
                     f"{single_thread_cycles} V-cycle(s) on one thread x {need}"}
    return out, nt


def run_reference(args, ws, rank):
    """The reference arm: one step = one V-cycle of the reference's own loop
    (oracle port of perform_vcycle, -march=native, all host threads) on the
    power-of-two twin, W warm-up cycles then K timed cycles of one solve from
    zero; solves/s = 1 / (mean timed cycle x the cycles the same run needed to
    reach 1e-10)."""
    if rank != 0:
        return 0
    from mps3d_b200 import workloads as W

    n = args.n
    os.environ.setdefault("MPS_ORACLE_NATIVE", "1")
    nt = reference_twin(n)
    p = W.plasma_poisson(nt)
    times, rel, need, _ = oracle_cpu_solve(p, max_cycles=args.warmup + args.steps, single_thread_cycles=0, tol=0.0)
    timed = times[args.warmup:] if args.steps > 0 else times
    t_cycle = float(np.mean(timed))
    reached = next((i + 1 for i, r in enumerate(rel) if r <= 1e-10), None)
    if reached is None:  # the run was too short to reach the tolerance: asymptotic rate of its last cycles
        rate = min(max(rel[-1] / rel[-2], 1e-6), 0.999) if len(rel) > 1 else 0.5
        reached = len(rel) + int(np.ceil(np.log(1e-10 / rel[-1]) / np.log(rate)))
        how = f"{reached} cycles to 1e-10 extrapolated from the last cycles' rate"
    else:
        how = f"{reached} cycles to 1e-10 measured in the same run"
    value = 1.0 / (t_cycle * reached)
    hc = host_cpu()
    sample = (f"{len(timed)} timed V-cycles (after {args.warmup}) of one solve from zero with the FP64 restatement of "
              f"perform_vcycle on the {nt}^3 power-of-two twin of the {n}^3 problem (the reference hierarchy cannot "
              f"coarsen {n}), {hc['threads']} OpenMP threads, {hc['build']}; {t_cycle:.3f} s/cycle x {how}")
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_cycle * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(n, {"reference_twin_cells": nt ** 3,
                                      "hierarchy": "reference CELL (l/2 integer division), RB-GS 2/2, GMRES bottom"}),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": hc["threads"], "kind": "port", "sample": sample,
                         "nproc": hc["nproc"], "cpu_model": hc["cpu_model"], "build": hc["build"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_rel_residual_history": rel,
    }
    print(json.dumps(out))
    return 0


# ---------------------------------------------------------------------------
def oracle_reference(p, krylov=False):
    """The FP64 oracle's solution of ``p`` (GEOM hierarchy, converged to
    1e-13), its right-hand side and fine-level rows: the checker of the GPU
    solutions reported beside each figure."""
    from oracle import oracle as orc

    mg = orc.RowsMG(p, hier=orc.HIER_GEOM)
    b = orc.build_rhs(p)
    if krylov:
        x, hist = mg.fgmres(b, m=30, maxit=200, tol=1e-13)
    else:
        x, hist = mg.solve(b, maxit=80, tol=1e-13)
    return x, b, mg.rows(0), float(hist[-1])


def vs_oracle(p, x_ghosted, ref):
    """Relative residual of a GPU solution evaluated by the oracle (its rows
    and right-hand side) and its relative error against the oracle's
    converged FP64 solution."""
    from oracle import oracle as orc

    x_ref, b, rows, _ = ref
    xi = np.ascontiguousarray(np.asarray(x_ghosted)[1:-1, 1:-1, 1:-1])
    rr = float(np.linalg.norm(b - orc.rows_apply(p, rows, xi)) / np.linalg.norm(b))
    err = float(np.linalg.norm(xi - x_ref) / np.linalg.norm(x_ref))
    return {"rel_res_by_oracle": rr, "rel_err_vs_oracle": err}


# ---------------------------------------------------------------------------
def colour_pass_bytes(cells, s, coeff_field):
    """Algorithmic bytes of one red-black colour pass (red/black split layout):
    read the other colour (N/2 words), read f of the colour (N/2), write the
    colour (N/2), plus the cell coefficient k of both colours (N) when the
    operator has one (FP64 k in the FP64 hierarchy, FP32 k in the mixed one)."""
    b = 1.5 * cells * s
    if coeff_field == 1:
        b += cells * s
    return b


def vcycle_bytes(levels_cells, s, coeff_field, nu=4):
    """Algorithmic bytes of one V-cycle: per level nu*2 colour passes, the
    fused residual+restriction (read u, f, k; write N/8) and the fused
    prolongation+correction (read N/8, read+write u)."""
    tot = 0.0
    for i, n in enumerate(levels_cells[:-1]):
        tot += 2 * nu * colour_pass_bytes(n, s, coeff_field)
        tot += (2 * n + (n if coeff_field == 1 else 0) + n / 8.0) * s
        tot += (2 * n + n / 8.0) * s
    return tot


def geom_level_cells(nx, ny, nz):
    """Cells per level of the geometric hierarchy (l/2 per direction, stop
    at <= 125 cells)."""
    lev, d = [], [nx, ny, nz]
    while True:
        lev.append(d[0] * d[1] * d[2])
        if lev[-1] <= 125:
            return lev
        d = [max(1, q // 2) for q in d]


def batch_bytes(probs, infos, s):
    """Algorithmic bytes of a batch of constant-coefficient solves: each
    problem's V-cycles (vcycle_bytes with words of s bytes) plus, per outer
    iteration and once before the first, the FP64 residual (read x and b,
    write r as s) and, per outer iteration, the FP64 update (read e, read and
    write x)."""
    tot = 0.0
    for p, i in zip(probs, infos):
        n = p.lx * p.ly * p.lz
        it = i["iters"]
        vc = i.get("vcycles") or 2 * it
        tot += vc * vcycle_bytes(geom_level_cells(p.lx, p.ly, p.lz), s, 0)
        tot += (it + 1) * (16 + s) * n + it * (16 + s) * n
    return tot


def timed_solves(dp, xg, h, steps, ws, init=None, **kw):
    """ms per solve (CUDA events on the solving stream, max over ranks) and the last info."""
    import torch

    from mps3d_b200 import solver

    def one():
        if init is None:
            xg.zero_()
        else:
            xg.copy_(init)
        _, info = solver.linsolve_dev(dp, xg, handle=h, **kw)
        if info["status"] != 0:
            raise RuntimeError(f"solve failed: {info} {h.last_error()}")
        return info

    for _ in range(3):
        one()
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        info = one()
    e1.record()
    torch.cuda.synchronize()
    return dist_max(e0.elapsed_time(e1), ws) / steps, info


def bench_poisson65(args, ws, rank, h, dev, deferred):
    """Plain FP64 Poisson, 65^3 cells on the unit cube, coefficient 1, Dirichlet
    0, U[-1,1] right-hand side, to 1e-10 relative residual: GPU solves/s (mixed
    and FP64) and, on rank 0 with one GPU, the oracle's restatement of the
    reference's V-cycle loop solving the 64^3 power-of-two twin on the host
    cores (the reference cannot coarsen 65)."""
    import torch

    from mps3d_b200 import solver, workloads as W

    p = W.poisson_dirichlet(65)
    dp = solver.DeviceProblem(p, device=f"cuda:{dev}")
    x = torch.zeros(p.ghost_shape, dtype=torch.float64, device=f"cuda:{dev}")
    out = {"workload": "Poisson 65^3, unit cube, coefficient 1, Dirichlet 0, U[-1,1] source, 1e-10 rel. residual",
           "unit": "solves/s"}
    check = rank == 0 and ws == 1 and not args.skip_oracle
    sols = {}
    for prec in ("mixed", "fp64"):
        ms, info = timed_solves(dp, x, h, args.steps, ws, precision=prec, tol=1e-10, maxit=60)
        out[prec] = {"value": ws * 1e3 / ms, "ms_per_solve": ms, "iters": info["iters"], "rel_res": info["rel_res"]}
        sols[prec] = x.cpu().numpy()

    def later():  # host-core work, after every GPU timing of the run
        if check:
            ref = oracle_reference(p)
            for prec in ("mixed", "fp64"):
                out[prec].update(vs_oracle(p, sols[prec], ref))
        if rank == 0 and ws == 1 and not args.skip_cpu:
            from oracle import oracle as orc

            q = W.poisson_dirichlet(64)
            t0 = time.perf_counter()
            _, rel, _ = orc.solve(q, maxit=40, tol=1e-10, tol_kind=1)
            t = time.perf_counter() - t0
            out["cpu_oracle_64"] = {"s_per_solve": t, "vcycles": int(len(rel)), "final_rel_res": float(rel[-1]),
                                    "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
                                    "kind": "port (restatement of perform_vcycle, CELL hierarchy, 64^3 twin)"}

    deferred.append(later)
    return out


def bench_sg_step(args, ws, h, phi_fine, dev, deferred, check=False):
    """Implicit SG electron step, 129^3: the potential is the 257^3 plasma
    Poisson solution injected onto 129^3; FGMRES(30) preconditioned by an FP32
    (mixed) or FP64 V-cycle, to 1e-10 relative residual."""
    import torch

    from mps3d_b200 import capi, solver, workloads as W

    p3 = W.electron_sg_step(129, phi=W.inject_potential(phi_fine.cpu().numpy(), 129))
    dp3 = solver.DeviceProblem(p3, device=f"cuda:{dev}")
    x3 = torch.zeros(p3.ghost_shape, dtype=torch.float64, device=f"cuda:{dev}")
    out = {"workload": "implicit electron drift-diffusion step 129^3, Scharfetter-Gummel faces, dt 1e-11 s, "
                       "periodic x/y, ZGRD z; potential = 257^3 plasma Poisson solution injected",
           "unit": "solves/s", "tol_rel_residual": 1e-10}
    sols = {}
    hbm_peak, _ = load_peaks()
    cells = p3.lx * p3.ly * p3.lz
    for prec in ("mixed", "fp64"):
        ms, info = timed_solves(dp3, x3, h, args.steps, ws, precision=prec, krylov="fgmres", restart=30,
                                tol=1e-10, maxit=60)
        out[prec] = {"value": ws * 1e3 / ms, "ms_per_solve": ms, "iters": info["iters"],
                     "rel_res": info["rel_res"]}
        sols[prec] = x3.cpu().numpy()
        # the finest-level colour pass of the preconditioner, live CUDA-event
        # times of one more solve: explicit rows (7 coefficients of the
        # colour's cells), the other colour, f, the write -- 5 words per cell
        # pair of word size s
        h.set_profile(True)
        h.get_profile(reset=True)
        timed_solves(dp3, x3, h, 1, ws, precision=prec, krylov="fgmres", restart=30, tol=1e-10, maxit=60)
        pr = h.get_profile(reset=True)
        h.set_profile(False)
        if pr.count[capi.PROF_SMOOTH] > 0:
            s_b = 4 if prec == "mixed" else 8
            us = 1e3 * pr.ms[capi.PROF_SMOOTH] / pr.count[capi.PROF_SMOOTH]
            gbs = 5.0 * s_b * cells / (us * 1e-6) / 1e9
            out[prec]["colour_pass"] = {"us": us, "per_solve": pr.count[capi.PROF_SMOOTH], "bytes": 5.0 * s_b * cells,
                                        "gbs": gbs, "frac": gbs / hbm_peak}

    def later():
        if check:
            ref = oracle_reference(p3, krylov=True)
            for prec in ("mixed", "fp64"):
                out[prec].update(vs_oracle(p3, sols[prec], ref))

    deferred.append(later)
    return out


def bench_batch(args, ws, rank, h, dev, deferred):
    """64 independent constant-coefficient Poisson solves, cubic sizes drawn
    from {33,49,65,97,129}, Dirichlet 0, U[-1,1] right-hand sides, to 1e-10
    relative residual: one batched mixed-precision call (every V-cycle step
    of all problems in one launch, the iteration loop in one CUDA graph)
    against 64 sequential FP64 solves (one handle per size, so no
    reallocation between them)."""
    import torch

    from mps3d_b200 import capi, solver, workloads as W

    allp = W.batch_poisson(64)
    # N ranks: a cost-balanced share of the 64 problems each (strong scaling)
    mine = partition_by_cost([p.lx * p.ly * p.lz for p in allp], ws)[rank]
    ps = [allp[i] for i in mine]
    dps = [solver.DeviceProblem(p, device=f"cuda:{dev}") for p in ps]
    xs = [torch.zeros(p.ghost_shape, dtype=torch.float64, device=f"cuda:{dev}") for p in ps]
    cells = sum(p.lx * p.ly * p.lz for p in allp)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def batched(prec):
        for x in xs:
            x.zero_()
        return solver.linsolve_batched_dev(dps, xs, handle=h, tol=1e-10, precision=prec, maxit=60)

    handles = {}

    def sequential(prec):
        infos = []
        for dp, x in zip(dps, xs):
            n = dp.prob.lx
            if n not in handles:
                handles[n] = capi.Handle(dev)
            x.zero_()
            _, info = solver.linsolve_dev(dp, x, handle=handles[n], tol=1e-10, precision=prec, maxit=60)
            infos.append(info)
        return infos

    out = {"workload": "64 Poisson problems, unit cube, cubic sizes from {33,49,65,97,129} (seeded), Dirichlet 0, "
                       "U[-1,1] right-hand sides, 1e-10 relative residual",
           "cells": cells, "unit": "solves/s"}
    check = ws == 1 and not args.skip_oracle
    sols = {}
    for name, fn, prec in (("batched_mixed", batched, "mixed"), ("batched_fp64", batched, "fp64"),
                           ("sequential_fp64", sequential, "fp64"), ("sequential_mixed", sequential, "mixed")):
        for _ in range(3):
            infos = fn(prec)
        barrier(ws)
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record()
        for _ in range(args.steps):
            infos = fn(prec)
        e1.record()
        torch.cuda.synchronize()
        ms = dist_max(e0.elapsed_time(e1), ws) / args.steps
        bad = [i for i in infos if i["status"] != 0]
        if bad:
            raise RuntimeError(f"{name}: {len(bad)} problems failed: {bad[0]}")
        every = gather_results(infos, mine, ws, rank, 64)
        if rank == 0:
            out[name] = {"value": 64 * 1e3 / ms, "ms_per_batch": ms,
                         "max_rel_res": max(i["rel_res"] for i in every),
                         "iters": sorted({i["iters"] for i in every})}
            if name.startswith("batched"):
                # algorithmic bytes of all 64 solves over the batch's time
                gbs = batch_bytes(allp, every, 4 if prec == "mixed" else 8) / (ms * 1e-3) / 1e9
                hbm_peak, _ = load_peaks()
                out[name].update({"hbm_gbs": gbs, "hbm_frac": gbs / hbm_peak})
        if check:
            sols[name] = [xx.cpu().numpy() for xx in xs]
    if rank == 0:
        out["batched_mixed_over_sequential_fp64"] = out["batched_mixed"]["value"] / out["sequential_fp64"]["value"]
        out["ranks"] = ws
        out["scaling"] = "strong (64 problems split across the ranks by cell count)"
    for hh in handles.values():
        hh.close()

    def later():  # the oracle's converged FP64 solution of every problem (N=1 only)
        if not check:
            return
        refs = [oracle_reference(pp) for pp in ps]
        for name, xl in sols.items():
            checks = [vs_oracle(pp, xx, rr) for pp, xx, rr in zip(ps, xl, refs)]
            out[name]["max_rel_res_by_oracle"] = max(c["rel_res_by_oracle"] for c in checks)
            out[name]["max_rel_err_vs_oracle"] = max(c["rel_err_vs_oracle"] for c in checks)

    deferred.append(later)
    return out


def bench_adjoint(args, ws, h, dev, deferred):
    """Electron-flux adjoint at 129^3: loss = electron flux through z = L
    after 5 implicit SG steps; gradients w.r.t. the electrode voltage and the
    FP32 mobility field (torch.autograd over the C ABI: transposed SG solves,
    operator VJP, symmetric Poisson adjoint).  Timed: one forward + backward;
    checked: central differences with h = 1e-4 relative."""
    import torch

    from mps3d_b200 import workloads as W
    from mps3d_b200.adjoint import ElectronFluxAdjoint

    case = W.electron_adjoint_case(129)
    model = ElectronFluxAdjoint(case, device=f"cuda:{dev}", handle=h, tol=1e-12)
    V = case["v_front"]
    mu = torch.from_numpy(case["mu"]).to(f"cuda:{dev}")
    for _ in range(2):
        L0, gV, gmu = model.gradient(V, mu)
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    steps = max(1, args.steps // 2)
    for _ in range(steps):
        L0, gV, gmu = model.gradient(V, mu)
    e1.record()
    torch.cuda.synchronize()
    ms = dist_max(e0.elapsed_time(e1), ws) / steps
    # central differences on the FP64 model (mobility perturbed in FP64)
    tight = ElectronFluxAdjoint(case, device=f"cuda:{dev}", handle=h, tol=1e-13)
    _, gV_t, gmu_t = tight.gradient(V, mu.double())  # FP64 mobility: the FP64 gradient
    mu64 = mu.double()
    f = lambda v, m: float(tight.loss(torch.tensor(v, dtype=torch.float64, device=mu.device), m))  # noqa: E731
    hv = 1e-4 * V
    fd_V = (f(V + hv, mu64) - f(V - hv, mu64)) / (2 * hv)
    d = torch.from_numpy(np.random.default_rng(5005).uniform(-1.0, 1.0, size=mu.shape)).to(mu.device) * mu64 * 1e-4
    fd_mu = (f(V, mu64 + d) - f(V, mu64 - d)) / 2.0
    an_mu = float((gmu_t.double() * d).sum())
    g64 = gmu_t.cpu()
    mu_cpu = mu.double().cpu()
    res = {}

    def later():
        if ws == 1 and not args.skip_oracle:
            # the same model over the FP64 oracle's solves and VJP on the host cores
            sys.path.insert(0, os.path.join(ROOT, "tests"))
            from adjoint_oracle import oracle_bvec, oracle_solve

            ref = ElectronFluxAdjoint(case, device="cpu", solve_fn=oracle_solve, bvec_fn=oracle_bvec)
            L_r, gV_r, gmu_r = ref.gradient(V, mu_cpu)
            res["vs_fp64_oracle_gradient"] = {
                "rel_err_loss": abs(L0 - L_r) / abs(L_r), "rel_err_dL_dV": abs(gV_t - gV_r) / abs(gV_r),
                "rel_err_dL_dmu": float((g64 - gmu_r).norm() / gmu_r.norm()),
                "note": "FP64 mobility on both sides; tolerance 1e-12 (GPU) / 1e-14 (oracle)"}

    deferred.append(later)
    res.update({"workload": "electron flux through z=L after 5 implicit SG steps, 129^3 (plasma Poisson potential with "
                        "electrode voltage V; mobility mu FP32 field); gradients w.r.t. V and mu",
            "unit": "gradients/s", "value": ws * 1e3 / ms, "ms_per_gradient": ms, "loss": L0,
            "dL_dV": gV, "fd_dL_dV": fd_V, "rel_err_V": abs(fd_V - gV_t) / abs(gV_t),
            "rel_err_mu_directional": abs(fd_mu - an_mu) / abs(an_mu),
            "fd_step": "1e-4 relative (V; every mobility cell along a random direction)"})
    return res


def bench_plasma_step(args, ws, dev, deferred, check=False):
    """The potential + electron part of one implicit step at 129^3 on the
    device (mps_plasma_step_dev: space-charge source, potential solve, E
    field, electron operator, SG electron solve, floor, ghosts), against what
    a host-assembled step moves over PCIe: the H2D of the five ghosted
    electron-operator fields (vel x3, dcoeff, source) that the on-device
    assembly replaces, timed from pinned memory."""
    import torch

    from mps3d_b200 import step as ST, workloads as W

    case = W.plasma_step_case(129)
    stp = ST.PlasmaStep(case, device=f"cuda:{dev}")
    phi0 = torch.zeros(case["eps"].shape, dtype=torch.float64, device=f"cuda:{dev}")
    ne0 = torch.from_numpy(case["n_e0"]).to(f"cuda:{dev}")
    phi, ne = phi0.clone(), ne0.clone()

    def one():
        phi.copy_(phi0)
        ne.copy_(ne0)
        return stp.step(phi, ne)

    for _ in range(3):
        one()
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        ip, ie = one()
    e1.record()
    torch.cuda.synchronize()
    ms = dist_max(e0.elapsed_time(e1), ws) / args.steps
    # the host-assembled alternative's extra copies: 5 ghosted fields H2D
    host = torch.empty((5,) + tuple(case["eps"].shape), dtype=torch.float64).pin_memory()
    devb = torch.empty_like(host, device=f"cuda:{dev}")
    devb.copy_(host, non_blocking=True)
    torch.cuda.synchronize()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record()
    for _ in range(3):
        devb.copy_(host, non_blocking=True)
    c1.record()
    torch.cuda.synchronize()
    h2d_ms = c0.elapsed_time(c1) / 3
    out = {"workload": "potential + electron part of one implicit step, 129^3 (plasma Poisson with a dielectric slab "
                       "and one ion species, SG electron step dt 1e-11 s), operator assembled on the device",
           "unit": "steps/s", "value": ws * 1e3 / ms, "ms_per_step": ms, "phi_iters": ip["iters"],
           "electron_iters": ie["iters"], "h2d_ms_avoided": h2d_ms,
           "h2d_bytes_avoided": int(host.numel() * 8)}
    phi_h, ne_h = phi.cpu().numpy(), ne.cpu().numpy()
    stp.close()

    def later():
        if check:
            from oracle import step_oracle as SO

            phi_o, _, _, _, _, ne_o = SO.plasma_step(case, case["n_e0"])
            rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
            out["rel_err_phi_vs_oracle"] = rel(phi_h, phi_o)
            out["rel_err_ne_vs_oracle"] = rel(ne_h, ne_o)

    deferred.append(later)
    return out


def run_ours(args, ws, rank, local):
    import torch

    from mps3d_b200 import capi, solver, workloads as W

    assert torch.cuda.is_available(), "bench needs a CUDA device"
    dev = local if ws > 1 else 0
    torch.cuda.set_device(dev)
    n = args.n
    p = W.plasma_poisson(n)
    dp = solver.DeviceProblem(p, device=f"cuda:{dev}")
    h = capi.Handle(dev)
    x = torch.zeros(p.ghost_shape, dtype=torch.float64, device=f"cuda:{dev}")
    common = dict(tol=1e-10, maxit=60)

    def solve(prec):
        x.zero_()
        _, info = solver.linsolve_dev(dp, x, handle=h, precision=prec, **common)
        if info["status"] != 0:
            raise RuntimeError(f"solve failed: {info} {h.last_error()}")
        return info

    # warm-up (also allocates the workspace of both precisions)
    for _ in range(max(args.warmup, 0)):
        solve("mixed")
        solve("fp64")
    torch.cuda.synchronize()

    def timed(prec, profile=False):
        h.set_profile(profile)
        h.get_profile(reset=True)
        barrier(ws)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        infos = []
        with ClockSampler(dev, args.clocks_out) as cs:
            e0.record()
            for _ in range(args.steps):
                infos.append(solve(prec))
            e1.record()
            torch.cuda.synchronize()
        barrier(ws)
        ms = e0.elapsed_time(e1)
        prof = h.get_profile(reset=True)
        h.set_profile(False)
        return dist_max(ms, ws), infos, cs.summary(), prof

    # the headline figures: graphs without profiling nodes
    ms_mixed, inf_mixed, clk, _ = timed("mixed")
    ms_fp64, inf_fp64, clk64, _ = timed("fp64")
    # the per-kernel roofline: the same solves again with CUDA events around
    # every finest-level launch (event-record nodes inside the replayed graphs)
    _, _, _, prof = timed("mixed", profile=True)
    _, _, _, prof64 = timed("fp64", profile=True)
    per_mixed = ms_mixed / args.steps
    per_fp64 = ms_fp64 / args.steps
    # the solutions of both precisions, compared with the oracle below
    sol = {}
    for prec in ("mixed", "fp64"):
        solve(prec)
        sol[prec] = x.cpu().numpy()
    value = ws * 1e3 / per_mixed
    fp64_value = ws * 1e3 / per_fp64

    lev = geom_level_cells(n, n, n)

    hbm_peak, peak_kind = load_peaks()
    # roofline of the dominant kernel: finest-level colour pass, mixed solve
    cells = n ** 3
    cf = 1 if prof.coeff_field == 1 else 0
    s32 = prof.precision_bytes or 4
    if prof.count[capi.PROF_SMOOTH] == 0 or prof64.count[capi.PROF_SMOOTH] == 0:
        raise RuntimeError("no finest-level colour-pass timings were recorded")
    cp_ms = prof.ms[capi.PROF_SMOOTH] / max(prof.count[capi.PROF_SMOOTH], 1)
    cp_bytes = colour_pass_bytes(cells, s32, cf)
    achieved = cp_bytes / (cp_ms * 1e-3) / 1e9
    cp64_ms = prof64.ms[capi.PROF_SMOOTH] / max(prof64.count[capi.PROF_SMOOTH], 1)
    achieved64 = colour_pass_bytes(cells, 8, cf) / (cp64_ms * 1e-3) / 1e9
    # whole-solve algorithmic GB/s (V-cycles + outer FP64 residual/update)
    it_m = inf_mixed[-1]["iters"]
    vc_m = inf_mixed[-1]["vcycles"]
    solve_bytes_m = vc_m * vcycle_bytes(lev, 4, cf) + (it_m + 1) * (3 * 8 + 4) * cells + it_m * (4 + 16) * cells
    it_d = inf_fp64[-1]["iters"]
    solve_bytes_d = it_d * vcycle_bytes(lev, 8, cf) + (it_d + 1) * 3 * 8 * cells
    gbs_m = solve_bytes_m / (per_mixed * 1e-3) / 1e9
    gbs_d = solve_bytes_d / (per_fp64 * 1e-3) / 1e9

    # ---- end to end through the host C ABI: host buffers in, solution out ----
    e2e = None
    if not args.skip_e2e:
        import ctypes as C

        o = solver.make_opts(precision="mixed", **common)
        g = solver._grid(p)
        bcc = (C.c_int * 6)(*p.bc)

        def host_arrays(pinned):
            if pinned:
                mk = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
                ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
                xz = torch.zeros(p.ghost_shape, dtype=torch.float64).pin_memory()
            else:  # ordinary (pageable) numpy arrays, as a Fortran caller passes
                mk = lambda a: np.ascontiguousarray(a).copy()  # noqa: E731
                ptr = lambda t: C.c_void_p(t.ctypes.data)  # noqa: E731
                xz = np.zeros(p.ghost_shape)
            dc, src, bcs = mk(p.dcoeff), mk(p.source), [mk(v) for v in p.bcvals]
            return dc, src, bcs, xz, ptr

        def timed_host(pinned):
            dc, src, bcs, xz, ptr = host_arrays(pinned)
            bcv = (C.c_void_p * 6)(*[ptr(t) for t in bcs])
            infos, spent = [], 0.0
            for it in range(args.steps + 1):
                xz[...] = 0  # a zero initial guess for every solve (outside the timed call)
                barrier(ws)
                t0 = time.perf_counter()
                info = capi.Info()
                st = h._lib.mps_linsolve(h.h, C.byref(g), 0, 1.0, None, ptr(dc), None, ptr(src), bcc, bcv, None,
                                         ptr(xz), C.byref(o), C.byref(info))
                dt_call = time.perf_counter() - t0
                if st != 0:
                    raise RuntimeError(f"host solve failed {st} {h.last_error()}")
                if it > 0:  # the first call is a warm-up
                    spent += dt_call
                    infos.append(info)
            return dist_max(spent, ws), infos, xz

        t_e2e, infos_h, x_host = timed_host(True)
        ghost = int(np.prod(p.ghost_shape)) * 8
        faces = sum(int(v.size) for i, v in enumerate(p.bcvals) if p.bc[i] in (1, 2)) * 8
        dev_ms = float(np.mean([i.time_ms for i in infos_h]))
        per_call = t_e2e / args.steps
        e2e = {"value": ws * args.steps / t_e2e, "unit": UNIT, "h2d_bytes_per_step": 3 * ghost + faces,
               "d2h_bytes_per_step": ghost, "ms_per_step": per_call * 1e3,
               "device_ms_per_step": dev_ms,
               "host_link_gbs": (4 * ghost + faces) / max(per_call - dev_ms * 1e-3, 1e-9) / 1e9,
               "buffers": "pinned host memory (page-locked)"}
        # check the host-path answer against the device-path answer
        dx = float(np.abs(x_host.numpy() - sol["mixed"]).max() / max(np.abs(sol["mixed"]).max(), 1e-300))
        if not args.skip_pageable:
            t_pg, _, _ = timed_host(False)
            e2e["pageable"] = {"value": ws * args.steps / t_pg, "unit": UNIT, "ms_per_step": t_pg / args.steps * 1e3,
                               "buffers": "pageable host memory (numpy arrays, as a Fortran caller passes)"}

    # ---- secondary configurations (figures beside the headline line); every
    # host-core computation (oracle checks, CPU baselines) is deferred until
    # all GPU timings of the run are done, so that no OpenMP thread of the
    # oracle competes with the thread that drives the GPU ----
    others = {}
    deferred = []
    if not args.skip_others and n == 257:
        check = rank == 0 and ws == 1 and not args.skip_oracle
        others["poisson_65"] = bench_poisson65(args, ws, rank, h, dev, deferred)
        others["sg_step_129"] = bench_sg_step(args, ws, h, x, dev, deferred, check=check)
        others["batch64"] = bench_batch(args, ws, rank, h, dev, deferred)
        others["adjoint_129"] = bench_adjoint(args, ws, h, dev, deferred)
        others["plasma_step_129"] = bench_plasma_step(args, ws, dev, deferred, check=check)

    # ---- CPU baseline: the oracle port on the host cores (rank 0, N=1) ----
    cpu = None
    if rank == 0 and ws == 1 and not args.skip_cpu:
        cpu, _ = cpu_baseline_figures(n, problem=p)

    # ---- parity of the reported solutions against the FP64 oracle (rank 0, N=1) ----
    parity = None
    if rank == 0 and ws == 1 and not args.skip_oracle:
        ref = oracle_reference(p)
        parity = {prec: vs_oracle(p, sol[prec], ref) for prec in ("mixed", "fp64")}
        parity["oracle_final_rel_res"] = ref[3]
        del ref
    for fn in deferred:
        fn()

    traffic = None
    tpath = os.path.join(ROOT, "profiles", "colour_pass_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        traffic = tj.get("bytes_per_launch_257")

    launches = inf_mixed[-1]["launches"]
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_mixed, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "mixed: f32 V-cycle, f64 residual/update", "data": "synthetic",
        "config": workload_config(n, {"iters_mixed": it_m, "vcycles_mixed": vc_m, "iters_fp64": it_d}),
        "fp64": {"value": fp64_value, "unit": UNIT, "ms_per_step": per_fp64, "dtype": "f64",
                 "hbm_gbs_solve": gbs_d, "clocks": clk64},
        "mixed_over_fp64": fp64_value and value / fp64_value,
        "hbm_gbs_solve": gbs_m,
        "hbm_frac_solve": gbs_m / hbm_peak,
        "fp64_hbm_frac_solve": gbs_d / hbm_peak,
        "roofline": {"bound": "hbm", "kernel": "finest-level red/black pass, FP32, mixed solve: k_colour_tma<float,4,6> "
                                               "(TMA-staged rows; the passes from a valid state) and "
                                               "k_colourv_split<float,4> (the black pass after each outer residual, "
                                               "which writes the red pass from zero itself), averaged",
                     "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                     "peak_kind": peak_kind, "traffic": traffic, "bytes_per_launch": cp_bytes,
                     "launch_ms": cp_ms, "fp64_achieved": achieved64, "fp64_frac": achieved64 / hbm_peak},
        "clocks": clk,
        "gpu_launches": launches * args.steps,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "final_rel_residual": inf_mixed[-1]["rel_res"],
        # the headline solutions checked by the FP64 oracle on the same inputs
        # (relative residual evaluated by the oracle; relative error against
        # its solve converged to 1e-13)
        "vs_oracle": parity,
        # live CUDA-event timings of the finest-level launches, per class:
        # launches per solve and microseconds per launch
        "finest_level_us": {
            name: {cls: {"per_solve": pr.count[ci] / args.steps,
                         "us": 1e3 * pr.ms[ci] / max(pr.count[ci], 1)}
                   for cls, ci in (("smooth", capi.PROF_SMOOTH), ("restrict", capi.PROF_RESTRICT),
                                   ("prolong", capi.PROF_PROLONG), ("resid", capi.PROF_RESID))}
            for name, pr in (("mixed", prof), ("fp64", prof64))},
        "other_configs": others,
    }
    if e2e is not None:
        out["e2e_vs_device_max_rel_diff"] = dx
    if rank == 0:
        print(json.dumps(out))
    h.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-oracle", action="store_true", help="no parity figures against the FP64 oracle")
    ap.add_argument("--skip-pageable", action="store_true", help="no end-to-end figure with pageable host buffers")
    ap.add_argument("--clocks-out", default=None, help="folder for the nvidia-smi clock samples (default: a temp file)")
    ap.add_argument("--skip-others", action="store_true", help="only the headline configuration")
    args = ap.parse_args()
    # CPU timings use the oracle built for this host's CPU (-march=native)
    os.environ.setdefault("MPS_ORACLE_NATIVE", "1")
    ws, rank, local = dist_init()
    try:
        if args.impl == "reference":
            return run_reference(args, ws, rank)
        return run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
