#!/usr/bin/env python
"""Element-assembly benchmark: elements/s per Newton assembly of the 3D quadratic Bezier hex
(NURBS3_Cube2, 27 nodes, 27 Gauss points) 32x32x64 mesh on a 0.05x0.05x0.1 m box, damaged Glen
viscoelastic ice (n=3, A Arrhenius at -10 degC), FP64 residual with an FP32 tangent (tensor cores, split operands, or CUDA cores),
next to the plain FP64 GPU assembly and the CPU oracle.

One step = one Newton assembly = Physics::Assemble of the displacement step followed by the
phase-field step (residual + tangent scattered into the device CSR, history updated).  The
displacement state alternates between two nearby fields so every assembly re-solves the return
map from a warm start, as consecutive Newton iterations do.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
Under torchrun each rank assembles its own copy of the mesh (weak scaling, no collective on the
data path); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "elements/s per Newton assembly & %HBM peak, mixed vs plain FP64 GPU"

# DRAM bytes (read + write) per launch of the tensor-core tangent on the 65,536-element hex workload, from the
# ncu capture summarised in profiles/dram_assembly_hex16x16x32.md (8,192-element case, scaled by the element count).
TC_TANGENT_DRAM_BYTES_FULL = 0.38e9 + 1.73e9
WORKLOAD = ("3D quadratic Bezier hex NURBS3_Cube2 32x32x64 (65,536 elements, 76,296 control points, "
            "27 ips), damaged Glen viscoelastic ice n=3 at -10 degC, u-step + phase-step assembly")


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix=f"icefem_clocks_{self.index}_", suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        with open(self.path) as f:
            lines = f.read().splitlines()
        os.unlink(self.path)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_bytes(mesh, nnz_u, nnz_p, tangent_bytes, hist_u=24, nnz_t=None):
    """Per-assembly algorithmic bytes: every array read or written once.  hist_u: doubles of displacement-step
    history per ip (24 for the viscoelastic family, 16 for linear elasticity); nnz_t: the temperature step's
    nonzeros when the configuration has one."""
    nel, nen, nn, dim = mesh.n_elems, mesh.nen, mesh.n_nodes, mesh.dim
    nh = nel * nen
    geo = nel * nen * 4 + nel * dim * 9 * 8 + nn * dim * 8 + (nn * 8 if dim == 3 else 0)
    points = geo + 2 * nn * dim * 8 + 2 * nn * 8 + nh * hist_u * 8       # U, Uold, phase, phase_old, history
    u_resid = nn * dim * 8
    u_csr = nnz_u * tangent_bytes
    phase = geo + nn * dim * 8 + 2 * nn * 8 + nh * 8 * 8 + nn * 8 + nnz_p * tangent_bytes
    out = {"u_points": points, "u_gather": u_resid + u_csr, "u_step": points + u_resid + u_csr,
           "phase_step": phase, "assembly": points + u_resid + u_csr + phase}
    if nnz_t is not None:      # T, T_old, dT/dt, viscous dissipation (current, old), residual, CSR values
        t_step = geo + 3 * nn * 8 + 2 * nh * 8 + nn * 8 + nnz_t * tangent_bytes
        out["t_step"] = t_step
        out["assembly"] += t_step
    return out


def tangent_flops(mesh):
    nU = mesh.dim * mesh.nen
    per_ip = 6 * 6 * nU * 2 + nU * nU * 6 * 2
    return mesh.n_elems * mesh.nen * per_ip


DT = {0: 1.0, 1: 100.0, 2: 10.0, 3: 100.0, 4: 100.0}      # time step of each configuration's assemblies
DU_DT = {2: 0.1}                                            # dT/dt scaling of the thermal step (configuration 2)


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def oracle_full_mesh(idx, nthreads, steps, warmup, budget_s=150.0, gpu_device=None, prec=None):
    """The oracle (CPU restatement, all host threads) on the FULL mesh of configuration `idx`: every staggered step
    of one Newton assembly per iteration, the displacement alternating between two nearby fields (as the GPU
    benchmark does).  Iterations stop early once `budget_s` of CPU time is spent.  With `gpu_device`, a fresh GPU
    context assembles the same state once and its residual / tangent errors against the oracle's first assembly
    are returned too.  Returns (elements/s, elements, median s per assembly, iterations timed, errors)."""
    from ice_fem_2025a_b200 import abi, config as cf
    from oracle import oracle as orc
    mesh, d, st = cf.config(idx)
    mats, opts = cf.materials(d), cf.options_from_json(d)
    if prec is not None:
        opts.tangent_precision = prec
    o = orc.context(mesh, mats, opts)
    s = st()
    cf.apply_state(o, s)
    U0 = s[0][abi.STATE_CUR]
    U1 = U0 * (1.0 + 1e-3)
    dt, du = DT[idx], DU_DT.get(idx, 0.0)
    errors = None
    if gpu_device is not None:
        g = abi.product_context(mesh, mats, opts, device=gpu_device)
        cf.apply_state(g, s)
        errors = {}
        for step in range(o.nsteps):
            o.assemble_mt(step, nthreads, dt=dt, du_dt=du)
            g.assemble(step, dt=dt, du_dt=du)
            f32 = opts.tangent_precision != abi.PREC_FP64
            errors[f"step{step}"] = {
                "residual_rel_err": _rel(g.residual(step), o.residual(step)),
                "tangent_frob_err": _rel(g.matrix_values(step, abi.F32 if f32 else abi.F64), o.matrix_values(step))}
        g.close()
        cf.apply_state(o, s)
    times = []
    t_start = time.perf_counter()
    for k in range(warmup + steps):
        o.set_state(0, abi.STATE_CUR, U1 if k % 2 else U0)
        t0 = time.perf_counter()
        for step in range(o.nsteps):
            o.assemble_mt(step, nthreads, dt=dt, du_dt=du)
        if k >= warmup:
            times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > budget_s and times:
            break
    o.close()
    med = statistics.median(times)
    return mesh.n_elems / med, mesh.n_elems, med, len(times), errors


def run_reference(args, rank, world):
    """The reference arm: the oracle port of the reference's assembly on the host cores, on the same full mesh as
    the GPU arm (rank 0 only under torchrun)."""
    if rank != 0:
        return 0
    nthreads = os.cpu_count() or 1
    eps, nel, med, n_timed, _ = oracle_full_mesh(args.config, nthreads, max(1, args.steps), min(args.warmup, 1))
    sample = (f"full {nel}-element mesh, every staggered step of one Newton assembly per step, median of {n_timed} "
              f"timed steps (of {args.steps} requested; the timed loop stops after 150 s)")
    line = {"impl": "reference", "metric": METRIC, "value": eps, "unit": "elements/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": med * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD if args.config == 1 else CONFIG_NAMES[args.config],
                       "elements": nel, "parallelism": "host threads"},
            "cpu_baseline": {"value": eps, "unit": "elements/s", "cores": nthreads, "kind": "port", "sample": sample},
            "e2e": {"value": eps, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


CONFIG_NAMES = {
    0: "2D B2_2 64x128 (8,192 elements), linear-elastic ice + AT2 phase field, u-step + phase step",
    1: WORKLOAD,
    2: "2D thermomechanical slab B2_2 512x256 (131,072 elements), damaged Glen ice, gravity, u + phase + T steps",
    3: "3D hex 48x48x48 (110,592 elements), damaged Glen ice, smooth random strain, u-step + phase step + adjoints",
    4: "256 batched 2D specimens (16x32 .. 96x192, 2,041,048 elements), per-specimen (Gc, l, A, n), u-step + phase "
       "step + adjoints replayed as one CUDA graph",
}


def config_report(idx, local, nthreads, steps=5, warmup=3):
    """Device throughput of one configuration (every staggered step of a Newton assembly; adjoints for 3 and 4),
    its HBM fraction, the plain FP64 comparator, and the oracle on the full mesh: CPU baseline and errors."""
    import torch
    from ice_fem_2025a_b200 import abi, config as cf
    mesh, d, st = cf.config(idx)
    mats, opts = cf.materials(d), cf.options_from_json(d)
    prec = abi.PREC_TC_SPLIT if mesh.dim == 3 else abi.PREC_FP32
    opts.tangent_precision = prec
    ctx = abi.product_context(mesh, mats, opts, device=local)
    state = st()
    cf.apply_state(ctx, state)
    dev = torch.device("cuda", local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    dt, du = DT[idx], DU_DT.get(idx, 0.0)
    n_mats = len(mats)
    adj = idx in (3, 4)

    def timed(fn):
        for _ in range(warmup):
            fn()
        for sidx in range(ctx.nsteps):
            ctx.sync(sidx)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        for sidx in range(ctx.nsteps):
            ctx.sync(sidx)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / steps

    def assembly():
        for sidx in range(ctx.nsteps):
            ctx.assemble_async(sidx, dt=dt, du_dt=du)

    out = {"workload": CONFIG_NAMES[idx], "elements": mesh.n_elems, "steps": steps, "warmup": warmup,
           "tangent": {abi.PREC_TC_SPLIT: "tc_split", abi.PREC_FP32: "fp32"}[prec]}
    ms = timed(assembly)
    info = [ctx.step_info(sidx) for sidx in range(ctx.nsteps)]
    hbm, _, peak_kind = measured_peaks()
    rheo_le = mats[0].rheology == abi.RHEO["LinearElastic"]
    ab = algorithmic_bytes(mesh, info[0][1], info[1][1], 4, hist_u=16 if rheo_le else 24,
                           nnz_t=info[2][1] if ctx.nsteps > 2 else None)
    out.update({"ms_per_assembly": ms, "elements_per_s": mesh.n_elems / (ms * 1e-3),
                "algorithmic_GB": ab["assembly"] / 1e9, "hbm_frac": ab["assembly"] / (ms * 1e-3) / 1e9 / hbm,
                "hbm_peak": f"{hbm} GB/s ({peak_kind})"})
    ctx.set_tangent(abi.TANGENT_REFERENCE, abi.PREC_FP64)
    ms64 = timed(assembly)
    ctx.set_tangent(abi.TANGENT_REFERENCE, prec)
    out["fp64_gpu"] = {"ms_per_assembly": ms64, "elements_per_s": mesh.n_elems / (ms64 * 1e-3),
                       "speedup_mixed_vs_fp64": ms64 / ms}
    if adj:
        if idx == 3:
            def adjoint():
                for sidx in (0, 1):
                    ctx.adjoint(sidx, dt=dt)
            ms_adj = timed(adjoint)
            out["adjoint"] = {"ms_per_adjoint_pair": ms_adj,
                              "note": "dR/d(Gc, l, A, n) of the u-step and the phase step, lambda^T dR per material set"}
        else:
            ctx.graph_capture([0, 1], with_adjoint=True, dt=dt)
            ms_graph = timed(ctx.graph_launch)
            out["graph"] = {"ms_per_replay": ms_graph, "elements_per_s": mesh.n_elems / (ms_graph * 1e-3),
                            "specimens": n_mats,
                            "note": "one CUDA-graph replay = u-step + phase step residual and tangent + their adjoints "
                                    "over all specimens"}
    ctx.close()
    eps, nel, med, n_timed, errors = oracle_full_mesh(idx, nthreads, 1, 0, budget_s=60.0, gpu_device=local, prec=prec)
    out["errors_vs_fp64_oracle"] = errors
    out["cpu_baseline"] = {"value": eps, "unit": "elements/s", "cores": nthreads, "kind": "port",
                           "sample": f"full {nel}-element mesh, one Newton assembly ({med:.2f} s)"}
    return out


def newton_report(device):
    """Staggered Newton solves (displacement-controlled tension, host direct linear solve) with the FP64 tangent
    and with the mixed-precision one: iterations per time step and the converged fields' difference."""
    from ice_fem_2025a_b200 import abi, config as cf, newton

    cases = (("2D B2_2 64x128 linear-elastic AT2, 3 load steps", 0, 1.0, abi.PREC_FP32, 1.0, 1.0e-3, 2.0e-4, False),
             ("3D hex 4x4x8 damaged Glen viscoelastic, 3 load steps, tight return map", 1, 0.125, abi.PREC_TC_SPLIT,
              1.0, 1.0e-4, 2.0e-5, True))
    out = []
    for name, idx, scale, prec, dt, s0, ds, tight in cases:
        runs = {}
        for p in (abi.PREC_FP64, prec):
            mesh, d, st = cf.config(idx, scale=scale)
            if tight:
                d["B200"]["ReturnMapTolerance"] = "tight"
            opts = cf.options_from_json(d)
            opts.tangent_precision = p
            ctx = abi.product_context(mesh, cf.materials(d), opts, device=device)
            cf.apply_state(ctx, st())
            H = float(np.ptp(mesh.coords[:, mesh.dim - 1]))
            solver = newton.StaggeredNewton(ctx, {0: newton.box_constraints(ctx, mesh, s0 * H)})
            its, fields, t0 = [], [], time.perf_counter()
            for k in range(3):
                logs = solver.solve_time_step(t=k * dt, dt=dt)
                its.append([lg.iterations for lg in logs] + [all(lg.converged for lg in logs)])
                fields.append([ctx.get_state(s, abi.STATE_CUR) for s in range(ctx.nsteps)])
                ctx.commit(2)
                solver.set_constraints({0: newton.box_constraints(ctx, mesh, (s0 + (k + 1) * ds) * H)})
            runs[p] = (its, fields, time.perf_counter() - t0)
            ctx.close()
        f64, fmx = runs[abi.PREC_FP64][1], runs[prec][1]
        err = max(float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
                  for ka, kb in zip(fmx, f64) for a, b in zip(ka, kb))
        out.append({"case": name, "mixed": {abi.PREC_FP32: "fp32", abi.PREC_TC_SPLIT: "tc_split"}[prec],
                    "iterations_fp64": runs[abi.PREC_FP64][0], "iterations_mixed": runs[prec][0],
                    "field_rel_err_mixed_vs_fp64": err,
                    "note": "iterations per time step: [u-step, phase step, converged]"})
    out.append(device_solve_report(device))
    return out


def device_solve_report(device):
    """The 2D 64x128 load steps with the linear solve on the device (GMRES; smoothed-aggregation multigrid set up
    once per time step for the u-step, node blocks for the phase step) against the host direct solve: wall time
    of the three time steps, Newton iterations and the converged fields' difference."""
    from ice_fem_2025a_b200 import abi, config as cf, newton

    res = {}
    for label, lin in (("host_superlu", newton.host_direct_solve), ("device_gmres_amg", newton.device_gmres_solve)):
        mesh, d, st = cf.config(0, scale=1.0)
        opts = cf.options_from_json(d)
        opts.tangent_precision = abi.PREC_FP32
        ctx = abi.product_context(mesh, cf.materials(d), opts, device=device)
        cf.apply_state(ctx, st())
        H = float(np.ptp(mesh.coords[:, mesh.dim - 1]))
        solver = newton.StaggeredNewton(ctx, {0: newton.box_constraints(ctx, mesh, 1.0e-3 * H)}, lin_solve=lin)
        its, fields, t0 = [], [], time.perf_counter()
        for k in range(3):
            if lin is newton.device_gmres_solve:
                ctx.set_preconditioner(0, abi.PC_AMG_REUSE)   # a new hierarchy per time step
            logs = solver.solve_time_step(t=k * 1.0, dt=1.0)
            its.append([lg.iterations for lg in logs] + [all(lg.converged for lg in logs)])
            fields.append([ctx.get_state(s, abi.STATE_CUR) for s in range(ctx.nsteps)])
            ctx.commit(2)
            solver.set_constraints({0: newton.box_constraints(ctx, mesh, (1.0e-3 + (k + 1) * 2.0e-4) * H)})
        res[label] = (its, fields, time.perf_counter() - t0)
        ctx.close()
    fh, fd = res["host_superlu"][1], res["device_gmres_amg"][1]
    err = max(float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)) for ka, kb in zip(fd, fh)
              for a, b in zip(ka, kb))
    return {"case": "2D B2_2 64x128 linear-elastic AT2, 3 load steps, FP32 tangent: linear solve on the host vs the device",
            "iterations_host_superlu": res["host_superlu"][0], "iterations_device": res["device_gmres_amg"][0],
            "wall_s_host_superlu": res["host_superlu"][2], "wall_s_device": res["device_gmres_amg"][2],
            "field_rel_err_device_vs_host": err,
            "note": "wall time of the three time steps (assembly, constraints, linear solves, state updates)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--prec", default="tc_split", choices=["fp32", "tc_split"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--slabs", type=int, default=8,
                    help="element slabs of the end-to-end u-step: each slab's rows are copied out while later slabs compute")
    ap.add_argument("--scale", type=float, default=1.0, help="shrink the mesh (profiling captures)")
    ap.add_argument("--no-newton", action="store_true", help="skip the Newton-iteration report")
    ap.add_argument("--no-configs", action="store_true", help="skip the report of the other four configurations")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    from ice_fem_2025a_b200 import abi, config as cf, replicas

    mesh, d, st = cf.config(args.config, scale=args.scale, seed=rank)
    mats, opts = cf.materials(d), cf.options_from_json(d)
    opts.tangent_precision = abi.PREC_TC_SPLIT if args.prec == "tc_split" else abi.PREC_FP32
    ctx = abi.product_context(mesh, mats, opts, device=local)
    state = st()
    cf.apply_state(ctx, state)
    nU, nnz_u = ctx.step_info(0)
    nP, nnz_p = ctx.step_info(1)
    dev = torch.device("cuda", local)
    U0 = torch.tensor(state[0][abi.STATE_CUR], dtype=torch.float64, device=dev)
    U1 = U0 * (1.0 + 1e-3)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    import ctypes as C
    setst = ctx.lib.ifem_set_state
    step_dt = DT[args.config]

    def set_u(k):
        src = U1 if k % 2 else U0
        ctx._check(setst(ctx.h, 0, abi.STATE_CUR, C.cast(src.data_ptr(), C.POINTER(C.c_double)), nU))

    def one_step(k):
        set_u(k)
        ctx.assemble_async(0, dt=step_dt)
        ctx.assemble_async(1, dt=step_dt)

    def timed(nsteps, launches_per_step=6):
        for k in range(args.warmup):
            one_step(k)
        ctx.sync(0); ctx.sync(1)
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(nsteps):
            one_step(k)
        e1.record(stream)
        ctx.sync(0); ctx.sync(1)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        return replicas.max_over_ranks(ms, dist, dev) / nsteps

    # ---- mixed precision (headline) ----
    clocks = ClockSampler(local)
    clocks.start()
    ms_mixed = timed(args.steps)
    clk = clocks.stop()
    # per-kernel device times (synchronous passes, library events)
    kern = {"u_points": [], "u_tangent": [], "u_gather": [], "phase_element": [], "phase_gather": []}
    rm_its = []
    for k in range(max(3, min(args.steps, 5))):
        set_u(k)
        ctx.assemble(0, dt=step_dt)
        s0 = ctx.stats(0)
        ctx.assemble(1, dt=step_dt)
        s1 = ctx.stats(1)
        kern["u_points"].append(s0.ms_points); kern["u_tangent"].append(s0.ms_tangent)
        kern["u_gather"].append(s0.ms_scatter); kern["phase_element"].append(s1.ms_element)
        kern["phase_gather"].append(s1.ms_scatter)
        rm_its.append(s0.rm_iterations)
    kern = {k: statistics.median(v) for k, v in kern.items()}
    # ---- plain FP64 GPU assembly ----
    ctx.set_tangent(abi.TANGENT_REFERENCE, abi.PREC_FP64)
    ms_fp64 = timed(args.steps)
    ctx.set_tangent(abi.TANGENT_REFERENCE, opts.tangent_precision)

    nel_job = mesh.n_elems * world
    value = nel_job / (ms_mixed * 1e-3)
    hbm, tc, peak_kind = measured_peaks()
    tb = 4
    ab = algorithmic_bytes(mesh, nnz_u, nnz_p, tb)
    dominant = max(kern, key=kern.get)
    flops = tangent_flops(mesh)
    if dominant == "u_tangent":
        ach = flops / (kern[dominant] * 1e-3) / 1e12
        full_tc = args.prec == "tc_split" and args.config == 1 and args.scale == 1.0
        roof = {"kernel": "u_tangent", "bound": "tensor", "achieved": ach, "peak": tc, "unit": "TFLOP/s",
                "frac": ach / tc, "traffic": TC_TANGENT_DRAM_BYTES_FULL if full_tc else None,
                "note": (f"dense-formulation tangent FLOP/s vs {peak_kind} bf16 peak; "
                         + ("tcgen05 kind::f16, FP16 hi/lo operands, three products per entry"
                            if args.prec == "tc_split" else "CUDA-core FP32 path"))}
    else:
        key = {"u_points": "u_points", "u_gather": "u_gather", "phase_element": "phase_step",
               "phase_gather": "phase_step"}[dominant]
        ach = ab[key] / (kern[dominant] * 1e-3) / 1e9
        roof = {"kernel": dominant, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "traffic": None, "note": f"algorithmic bytes of {key} / kernel time; peak {peak_kind}"}
    assembly_gbs = ab["assembly"] / (ms_mixed * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "elements/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 residual / f32 tangent" if args.prec == "fp32" else "f64 residual / f32-accurate tangent from f16 hi/lo tensor-core products",
        "data": "synthetic (seeded smooth strain field, seeded phase field)",
        "config": {"workload": WORKLOAD, "elements": mesh.n_elems, "nnz_u": nnz_u, "nnz_phase": nnz_p,
                   "l2": "inputs larger than L2 (no flush needed)", "parallelism": f"{world} independent replica(s)"},
        "hbm_frac_assembly": assembly_gbs / hbm, "assembly_algorithmic_GBps": assembly_gbs,
        "fp64_gpu": {"value": nel_job / (ms_fp64 * 1e-3), "ms_per_step": ms_fp64,
                     "hbm_frac": algorithmic_bytes(mesh, nnz_u, nnz_p, 8)["assembly"] / (ms_fp64 * 1e-3) / 1e9 / hbm},
        "speedup_vs_fp64_gpu": ms_fp64 / ms_mixed,
        "kernels_ms": kern, "rm_iterations_per_u_assembly": statistics.median(rm_its),
        "roofline": roof, "clocks": clk, "gpu_launches": 6 * args.steps,
    }
    # ---- end to end through the C-ABI with host buffers ----
    if not args.no_e2e:
        pin = lambda n, dt: torch.empty(n, dtype=dt, pin_memory=True).numpy()
        hU0 = pin(nU, torch.float64); hU0[:] = U0.cpu().numpy()
        hU1 = pin(nU, torch.float64); hU1[:] = U1.cpu().numpy()
        hP = pin(nP, torch.float64); hP[:] = state[1][abi.STATE_CUR]
        fU, fP = pin(nU, torch.float64), pin(nP, torch.float64)
        kU, kP = pin(nnz_u, torch.float32), pin(nnz_p, torch.float32)
        e2e_steps = max(2, min(args.steps, 5))
        ctx.set_readback_slabs(args.slabs)
        ms_slabbed = timed(args.steps)   # the same assembly on the device alone, in slabs

        def e2e_step(k):
            ctx.set_state(0, abi.STATE_CUR, hU1 if k % 2 else hU0)
            ctx.set_state(1, abi.STATE_CUR, hP)
            ctx.assemble_async(0, dt=step_dt)
            ctx.assemble_async(1, dt=step_dt)
            ctx.matrix_into(0, kU); ctx.residual_into(0, fU)
            ctx.matrix_into(1, kP); ctx.residual_into(1, fP)
            ctx.sync(0); ctx.sync(1)

        for k in range(2):
            e2e_step(k)
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(e2e_steps):
            e2e_step(k)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / e2e_steps
        ms = replicas.max_over_ranks(ms, dist, dev)
        line["e2e"] = {"value": nel_job / (ms * 1e-3), "unit": "elements/s", "ms_per_step": ms,
                       "h2d_bytes_per_step": (nU + nP) * 8, "d2h_bytes_per_step": (nU + nP) * 8 + (nnz_u + nnz_p) * 4,
                       "readback_slabs": args.slabs, "device_ms_per_step_slabbed": ms_slabbed,
                       "note": "state H2D from pinned host memory, residual + FP32 CSR values D2H to pinned host memory; "
                               "the u-step runs in element slabs whose rows are copied out while later slabs compute"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the oracle on the same full mesh: CPU baseline, and the GPU's errors against it on one fresh assembly
        nthreads = os.cpu_count() or 1
        eps, nel_s, med, n_timed, errors = oracle_full_mesh(args.config, nthreads, 2, 0, budget_s=60.0,
                                                            gpu_device=local, prec=opts.tangent_precision)
        line["cpu_baseline"] = {"value": eps, "unit": "elements/s", "cores": nthreads, "kind": "port",
                                "sample": f"oracle u-step + phase step on the full {nel_s}-element mesh, median of "
                                          f"{n_timed} ({med:.2f} s each)"}
        line["errors_vs_fp64_oracle"] = errors
        line["residual_rel_err"] = max(e["residual_rel_err"] for e in errors.values())
        line["tangent_frob_err"] = max(e["tangent_frob_err"] for e in errors.values())
    if rank == 0 and world == 1 and not args.no_configs:
        nthreads = os.cpu_count() or 1
        line["configs"] = {str(i): config_report(i, local, nthreads) for i in (0, 2, 3, 4)}
    if rank == 0 and not args.no_newton:
        line["newton"] = newton_report(local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
