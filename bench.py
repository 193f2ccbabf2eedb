"""Benchmark of the quasi-dynamic time-step path on B200.

Workload: the 401x401 linear-elastic quasi-dynamic strike-slip problem on a
grid stretched toward the fault and the surface, slip law, per-node
lognormal Dc (seeded synthetic inputs written in the reference's .in format,
loaded by the library's C++ reader), started from the reference's
steady-state initial guess and integrated with adaptive RK32.

A step is one accepted RK32 time step (its stage d_dt evaluations, each an
elliptic solve + fault update, plus rejected attempts).  ``value`` is whole-
job stage-solves per second (one stage-solve = one d_dt evaluation);
``sim_years_per_hour`` is reported beside it over the same window.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

The line also carries ``cycle``: three quasi-dynamic / fully dynamic cycles
of the 801x801 constant-grid workload (wall time, simulated years per hour,
event times, wave-equation steps per second), and ``response_mode``: the same
steps as ``value`` with the fault stress from the precomputed fault response.

Under torchrun (N > 1) every rank integrates its own replica (weak scaling,
no data-path collective); the timed region is bracketed by barriers and the
reported time is the max over ranks.
"""
import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "sim-years/hour & stage-solves/s: mixed+batched vs FP64 GPU, V err<=1e-6"
YEAR = 31557600.0
WORKLOAD = ("slip_var_401: linear-elastic quasi-dynamic, 401x401 SBP order 4 on a tanh-stretched grid "
            "(beta 2) over 30x30 km, slip law, lognormal Dc (mean 8 mm, sigma_ln 0.2), RK32 tol 1e-7, "
            "steady-state initial guess")


def _peaks():
    try:
        return json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, gpu_index=0):
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), "scy_clocks_%d.csv" % os.getpid())
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return None, 0, 1, 0
    import torch.distributed as dist
    import datetime
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return dist, rank, world, local


def _max_over_ranks(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _sum_over_ranks(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def make_workload(workdir, n=401, seed=0):
    from scycle_b200.configs import slip_var_401
    return slip_var_401(workdir, seed=seed, Ny=n, Nz=n, years=1.0e4)


def _fixture(name):
    path = os.path.join(HERE, "tests", "golden", "parity_%s.npz" % name)
    return np.load(path) if os.path.exists(path) else None


PARITY_FIELDS = ("slip", "slipVel", "psi", "tauP", "surfDisp")


def _field_errors(view, fx, k):
    """Norm-wise relative error per field, max |device - oracle| / max |oracle|."""
    return {f: float(np.max(np.abs(view.field(f) - fx[f][k])) / max(np.max(np.abs(fx[f][k])), 1e-300))
            for f in PARITY_FIELDS}


PARITY_RTOL = 1e-15  # solve tolerance of the parity legs (the stress is read from the solution)


def oracle_errors(name, make, rtol=PARITY_RTOL, batch_precision=None):
    """Error of the device path against the FP64 oracle: the driver (or a
    one-instance batch when ``batch_precision`` is given) forced onto the
    oracle's attempt sequence of the committed fixture
    tests/golden/parity_<name>.npz, fields compared after every recorded
    step; the maximum relative error per field.  The root finder takes the
    reference's Newton path (its derivative expression, fault.cpp:1051), as
    the oracle does."""
    fx = _fixture(name)
    if fx is None:
        return None
    work = tempfile.mkdtemp(prefix="scy_err_")
    att = list(zip(fx["attempt_dt"].tolist(), fx["attempt_acc"].astype(bool).tolist()))
    worst = {}
    if batch_precision is None:
        from scycle_b200.qd import QD
        q = QD.from_in(make(work), solve_rtol=rtol, exact_jacobian=False)
        q.force_attempts(att)
        q.integrate_begin_from_in()
        step = lambda n: q.integrate_steps(n)
        view, closer = q, q.close
    else:
        from scycle_b200.batch import Batch
        b = Batch([make(work)], solve_rtol=rtol, precision=batch_precision, exact_jacobian=False)
        view = b.instance(0)
        view.force_attempts(att)
        step = lambda n: b.run(n)
        closer = b.close
    done = 0
    for k, st in enumerate(fx["snap_steps"].tolist()):
        step(st - done)
        done = st
        for f, e in _field_errors(view, fx, k).items():
            worst[f] = max(worst.get(f, 0.0), e)
    closer()
    spread = {f: float(np.max(fx["spread_" + f])) for f in PARITY_FIELDS if "spread_" + f in fx.files}
    return {"steps": int(done), "solve_rtol": rtol, "max_rel_err": worst, "oracle_spread": spread,
            "norm": "max |device - oracle| / max |oracle| per field, maximum over the recorded steps",
            "fixture": "tests/golden/parity_%s.npz (oracle run free, device forced onto its attempts); "
                       "oracle_spread: the oracle against itself with plain instead of refined direct solves "
                       "on the same attempts (rounding-level differences carried by the integration)" % name}


# ---------------------------------------------------------------------------
ZT_DESC = ("ozk_gemm_kernel (z transforms of the preconditioner on the integer tensor cores: tcgen05 kind::i8 "
           "digit-plane products, TMA-fed, tensor-memory accumulators; two per apply)")
ZS_DESC = "ozk_split_reg_kernel (digit planes of the z-transform operand, the row held in registers; two per apply)"
BATCH_WORKLOAD = ("slip_var_401 ensemble: %d instances per GPU of the 401x401 stretched-grid slip-law workload "
                  "(seeds differ: lognormal Dc and initial state), every instance with its own RK32 step control")


def batch_config(args, world):
    """The workload description shared by both arms of the headline line."""
    return {"workload": BATCH_WORKLOAD % args.batch, "Ny": args.n, "Nz": args.n, "integrator": "RK32",
            "instances_per_gpu": args.batch, "parallelism": "replicas x%d" % world}


def run_batched(args, dist, rank, world, local):
    """The batched ensemble: args.batch instances of the workload per GPU
    advanced together (one CUDA graph launch per round of attempts).  A step
    is one scy_batch_run(1): every instance advances one accepted step."""
    import torch
    from scycle_b200 import _lib as S
    from scycle_b200.batch import Batch
    from scycle_b200.qd import QD
    L = S.lib()
    K = args.batch
    work = tempfile.mkdtemp(prefix="scy_batch_")
    paths = [make_workload(os.path.join(work, "i%d" % s), n=args.n, seed=rank * K + s) for s in range(K)]
    t0 = time.perf_counter()
    b = Batch(paths, solve_rtol=args.rtol, precision=args.batch_precision, transform_planes=args.transform_planes)
    setup_s = time.perf_counter() - t0
    for i in range(K):
        b.instance(i).record_attempts(True)
    b.run(args.warmup)
    torch.cuda.synchronize()

    def totals():
        st = [b.instance(i).integrate_steps(0) for i in range(K)]
        return sum(x.d_dt_evals for x in st), sum(x.t for x in st)

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = Clocks(local) if rank == 0 else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, s0 = totals()
    st0 = b.run(0)
    l0 = L.scy_launch_count()
    torch.cuda.nvtx.range_push("batched_timed")
    ev0.record()
    for _ in range(args.steps):
        st1 = b.run(1)
    ev1.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = L.scy_launch_count() - l0
    clk = clocks.stop() if clocks else None
    ms = _max_over_ranks(dist, ev0.elapsed_time(ev1))
    e1, s1 = totals()
    evals = _sum_over_ranks(dist, e1 - e0)
    sim_years = _sum_over_ranks(dist, (s1 - s0) / YEAR)
    out = {"value": evals / (ms / 1e3), "ms_per_step": ms / args.steps, "sim_years_per_hour": sim_years / (ms / 3.6e6),
           "sim_years_timed": sim_years, "stage_solves": evals, "instances": K * world, "setup_s": setup_s,
           "rounds": st1.rounds - st0.rounds, "redo_rounds": st1.redo_rounds - st0.redo_rounds,
           "cg_its": st1.cg_its, "groups": st1.groups, "gpu_launches": int(launches), "clocks": clk,
           "precision": args.batch_precision, "autotune": b.tuning(0)}
    # slip velocity against the plain FP64 single-instance path on instance 0's
    # own attempt sequence (the reported error of the batched form)
    if rank == 0:
        q = QD.from_in(paths[0], solve_rtol=args.rtol, precision="fp64")
        q.force_attempts(b.instance(0).attempts())
        q.integrate_begin_from_in()
        q.integrate_steps(args.warmup + args.steps)
        v_ref, v_b = q.field("slipVel"), b.instance(0).field("slipVel")
        out["v_rel_err_vs_fp64_single"] = float(np.max(np.abs(v_b - v_ref) / np.abs(v_ref)))
        q.close()
        # against the FP64 oracle: instance 0's workload (seed 0) forced onto
        # the oracle's first 100 attempts, through the same batched kernels
        if args.n == 401:
            e = oracle_errors("c1", lambda w: make_workload(w, n=401, seed=0), args.rtol,
                              batch_precision=args.batch_precision)
            out["oracle_error"] = e
            out["v_rel_err_vs_fp64_oracle"] = e["max_rel_err"]["slipVel"] if e else None
    # roofline of the batch's main kernels: a separate pass with the round's
    # launches issued directly and CUDA events around each launch
    b.set_graphs(False)
    b.profile(True)
    b.run(min(args.steps, 10))
    torch.cuda.synchronize()
    b.profile(False)
    peak = _peaks().get("hbm_gbs")
    peak_src = "measured"
    if peak is None:
        peak, peak_src = 6650.0, "fallback"
    # DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of
    # ncu captures of these kernels at 32 instances of the 401 x 401 workload
    # (profiles/batched_ensemble_kernels_401x401.md,
    # profiles/ozk_gemm_kernel_S5_12832x401x401.md,
    # profiles/b_full_kernel_32x401x401.md); other sizes report none
    sep = b.tuning(0)["operator_form"] != "cross"
    traffic = {"ysolve": 65362176.0, "ztransform": 28774656.0} if (args.batch == 32 and args.n == 401) else {}
    if args.batch == 32 and args.n == 401:
        traffic.update({"matvec": 99618816.0, "residual": 98234880.0} if sep else
                       {"matvec": 178643456.0, "residual": 187187968.0})
    opk = "b_full_kernel<%d> (separable form: 1D coefficient tables, register window along y)" if sep else \
        "b_cross_kernel<%d> (cross form: 33 coefficient planes)"
    kern = {}
    for nm, desc in (("ysolve", "b_ysolve_tma_kernel (banded Cholesky sweeps along y of the preconditioner)"),
                     ("matvec", (opk % 1) + ", CG operator application, p update fused"),
                     ("residual", (opk % 0) + ", initial residual of each stage solve"),
                     ("ztransform", ZT_DESC), ("zsplit", ZS_DESC)):
        pm, pl, pb = b.profile_collect(nm)
        if pl:
            us = pm / pl * 1e3
            ach = (pb / pl) / (us / 1e6) / 1e9
            kern[nm] = {"kernel": desc, "bound": "hbm", "unit": "GB/s", "peak": peak, "launch_us": us,
                        "algorithmic_bytes_per_launch": pb / pl, "achieved": ach, "frac": ach / peak,
                        "total_ms": pm, "launches": pl, "traffic": traffic.get(nm)}
    if "ztransform" in kern:
        # tensor-bound: algorithmic 8-bit integer operations of the digit
        # products (2 per multiply-add, S(S+1)/2 products of rows x Nz x Nz)
        # against the int8 dense rate, taken as twice the measured bf16 GEMM
        # rate (the nominal B200 ratio)
        S = args.transform_planes or (5 if args.batch_precision == "fp64" else 4 if args.batch_precision == "mixed"
                                      else 3)
        ops = 2.0 * S * (S + 1) / 2 * (args.n * K) * args.n * args.n
        bf16 = _peaks().get("bf16_tflops")
        tpeak, tsrc = (2.0 * bf16, "2 x measured bf16") if bf16 else (2.0 * 1590.0, "2 x fallback bf16 1590")
        k = kern["ztransform"]
        hbm_frac = k["frac"]
        k.update({"bound": "tensor", "unit": "TOP/s (int8)", "achieved": ops / (k["launch_us"] * 1e-6) / 1e12,
                  "peak": tpeak, "peak_source": tsrc, "planes": S, "int8_ops_per_launch": ops,
                  "fp64_equivalent_TFLOPs": 2.0 * (args.n * K) * args.n * args.n / (k["launch_us"] * 1e-6) / 1e12,
                  "hbm_frac_of_algorithmic_bytes": hbm_frac})
        k["frac"] = k["achieved"] / tpeak
    b.profile_clear()
    b.set_graphs(True)
    if kern:
        tot = sum(k["total_ms"] for k in kern.values())
        for k in kern.values():
            k["share_of_timed_kernels"] = k["total_ms"] / tot if tot else None
        top = max(kern, key=lambda k: kern[k]["total_ms"])
        t = kern[top]
        out["roofline"] = {"kernel": t["kernel"], "bound": t["bound"], "achieved": t["achieved"], "peak": t["peak"],
                           "unit": t["unit"], "frac": t["frac"], "peak_source": t.get("peak_source", peak_src),
                           "traffic": t["traffic"],
                           "launch_us": t["launch_us"], "algorithmic_bytes_per_launch": t["algorithmic_bytes_per_launch"],
                           "kernels": kern,
                           "note": "CUDA events on the launching stream in a pass with the round's launches issued "
                                   "directly; the dominant kernel is the one with the largest total time"}
    # end to end through the C ABI: every step the states go host -> device and
    # psi, slip and slip velocity device -> host (pinned buffers).  A fresh
    # batch of the same instances with the same warm-up, so the timed steps
    # cover the same simulated window as the device-timed ones (later steps
    # of this workload cost more: the instances approach their first events)
    b.close()
    b = Batch(paths, solve_rtol=args.rtol, precision=args.batch_precision, transform_planes=args.transform_planes)
    b.run(args.warmup)
    torch.cuda.synchronize()
    pin = lambda n: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    nst = b.state_size()
    nz_tot = sum(b.instance(i).Nz for i in range(K))
    hs = {"state": pin(nst), "psi": pin(nz_tot), "slip": pin(nz_tot), "vel": pin(nz_tot)}
    offs = np.cumsum([0] + [b.instance(i).Nz for i in range(K)])
    b.fault_field("psi", hs["psi"])
    b.fault_field("slip", hs["slip"])

    # positions of every instance's psi and slip in the state array
    # (instance i: psi then slip, Nz values each)
    pos_psi = np.concatenate([2 * offs[i] + np.arange(offs[i + 1] - offs[i]) for i in range(K)])
    pos_slip = pos_psi + np.repeat(np.diff(offs), np.diff(offs))

    def pack():
        hs["state"][pos_psi] = hs["psi"]
        hs["state"][pos_slip] = hs["slip"]

    pack()

    def e2e_step():
        b.set_states(hs["state"])
        b.run(1)
        b.fault_field("psi", hs["psi"])
        b.fault_field("slip", hs["slip"])
        b.fault_field("slipVel", hs["vel"])
        pack()

    if dist:
        dist.barrier()
    e0, _ = totals()
    t_w = time.perf_counter()
    ev0.record()
    for _ in range(args.steps):
        e2e_step()
    ev1.record()
    torch.cuda.synchronize()
    e_ms = _max_over_ranks(dist, ev0.elapsed_time(ev1))
    e1, _ = totals()
    out["e2e"] = {"value": _sum_over_ranks(dist, e1 - e0) / (e_ms / 1e3), "unit": "stage-solves/s",
                  "h2d_bytes_per_step": nst * 8, "d2h_bytes_per_step": 3 * nz_tot * 8,
                  "wall_s": time.perf_counter() - t_w}
    b.close()
    return out


C0_WORKLOAD = ("aging_const_101: linear-elastic quasi-dynamic, 101x101 SBP order 4 on a constant grid over 30x30 km, "
               "aging law, psi = 0.6 + N(0, 1e-4), RK32 atol 1e-7, the whole 200 simulated years")


def run_c0(args):
    """The CPU-runnable configuration end to end: the whole 200-year run on
    the device (plain FP64 driver), its error against the oracle on the
    oracle's own attempt sequence, and the oracle's run of the same 200
    years timed on one host core."""
    import torch
    from scycle_b200.configs import aging_const_101
    from scycle_b200.qd import QD
    work = tempfile.mkdtemp(prefix="scy_c0_")
    q = QD.from_in(aging_const_101(work, seed=0), solve_rtol=args.rtol)
    q.integrate_begin_from_in()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = q.integrate_steps(10 ** 8)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    q.close()
    out = {"workload": C0_WORKLOAD, "steps": st.step_count, "stage_solves": st.d_dt_evals, "wall_s": wall,
           "sim_years": st.t / YEAR, "sim_years_per_hour": (st.t / YEAR) / (wall / 3600.0),
           "stage_solves_per_s": st.d_dt_evals / wall,
           "oracle_error": oracle_errors("c0", lambda w: aging_const_101(w, seed=0))}
    if not args.no_cpu_baseline:
        r = oracle_on_all_cores("c0", 10 ** 8, max_workers=1)
        out["cpu_oracle_one_core"] = {"wall_s": r["timed_s_max"], "stage_solves": r["stage_solves"],
                                      "sim_years_per_hour": r["sim_years_per_hour"], "cpu_model": r["cpu_model"],
                                      "kind": "port", "note": "the whole 200-year run, one single-threaded instance"}
        out["gpu_over_cpu_sim_years"] = out["sim_years_per_hour"] / r["sim_years_per_hour"]
    return out


C3_WORKLOAD = ("pl_ensemble_c3: %d power-law viscoelastic instances (dislocation creep A=1e-4 MPa^-n/s, n=3, "
               "Q=135 kJ/mol, geotherm gradient U(15,30) K/km per instance, a-b perturbed by a Gaussian random "
               "field of std 0.002 and correlation length 2 km), grid sizes 101^2/201^2/301^2 in thirds, RK43")


def run_ensemble_c3(args, dist, rank, world, local):
    """The power-law ensemble of mixed grid sizes as one batch (one operator
    group per size, the groups on concurrent streams inside each round's
    graph).  A step is one scy_batch_run(1)."""
    import torch
    from scycle_b200.batch import Batch
    from scycle_b200.configs import pl_ensemble_c3
    from scycle_b200.ensemble import imbalance, instance_cost, partition
    work = tempfile.mkdtemp(prefix="scy_c3_")
    # one ensemble for the whole job (the same seed on every rank), split
    # over the ranks by estimated cost (grid size x stage solves)
    paths_all = pl_ensemble_c3(work, n_inst=args.c3, seed=0)
    costs = [instance_cost(p) for p in paths_all]
    shares = partition(costs, world)
    paths = [paths_all[i] for i in shares[rank]]
    t0 = time.perf_counter()
    b = Batch(paths, solve_rtol=args.rtol, precision=args.batch_precision)
    setup_s = time.perf_counter() - t0
    b.run(args.warmup)
    torch.cuda.synchronize()

    def totals():
        st = [b.instance(i).integrate_steps(0) for i in range(b.n)]
        return sum(x.d_dt_evals for x in st), sum(x.t for x in st)

    steps = max(1, args.c3_steps)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, s0 = totals()
    st0 = b.run(0)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(steps):
        st1 = b.run(1)
    ev1.record()
    torch.cuda.synchronize()
    ms = _max_over_ranks(dist, ev0.elapsed_time(ev1))
    e1, s1 = totals()
    out = {"workload": C3_WORKLOAD % args.c3, "instances": len(paths_all), "groups": st1.groups, "steps": steps,
           "partition": {"rule": "largest estimated cost first to the least-loaded rank", "ranks": world,
                         "instances_per_rank": [len(x) for x in shares], "cost_imbalance": imbalance(costs, shares)},
           "scaling": "strong (one ensemble split over the ranks)",
           "value": _sum_over_ranks(dist, e1 - e0) / (ms / 1e3), "unit": "stage-solves/s",
           "ms_per_step": ms / steps, "sim_years_per_hour": _sum_over_ranks(dist, (s1 - s0) / YEAR) / (ms / 3.6e6),
           "setup_s": setup_s, "cg_its": st1.cg_its, "rounds": st1.rounds - st0.rounds,
           "redo_rounds": st1.redo_rounds - st0.redo_rounds, "precision": args.batch_precision}
    b.close()
    if rank == 0 and not args.no_pl_ss:
        out["steady_state_guess_1e30"] = run_pl_steady_state()
    return out


def run_pl_steady_state():
    """The power-law steady-state initial guess at the reference's default
    viscosity cap (maxEffVisc = 1e30) for one instance of each grid size of
    the power-law ensemble (geotherm 22.5 K/km, seed 0): the effective-
    viscosity iteration with a direct solve of the non-separable viscosity
    operator per iteration (block Cholesky with double-double defect
    correction), timed end to end."""
    import torch
    from scycle_b200.configs import make_pl_problem
    from scycle_b200.qd import QD
    res = []
    for n in (101, 201, 301):
        work = tempfile.mkdtemp(prefix="scy_plss_")
        path = make_pl_problem(work, Ny=n, Nz=n, grad=22.5, extra={"guessSteadyStateICs": "1", "maxDeltaT": "1e6"})
        q = QD.from_in(path, solve_rtol=1e-12)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        q.integrate_begin_from_in()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        its, err, _ = q.steady_state_info()
        tr = q.steady_state_trace()
        eff = q.field("effVisc")
        res.append({"n": n, "wall_s": wall, "iterations": its, "last_change": err,
                    "corrections": int(tr[:, 0].sum()), "max_rel_residual": float(tr[:, 2].max()),
                    "effVisc_decades": float(np.log10(eff.max() / eff.min()))})
        q.close()
    return {"cases": res, "note": "set-up (once per run); the time-step operator of the power-law driver is "
                                  "built on the shear modulus (powerLaw.cpp:1110-1113), the viscosity enters "
                                  "through the viscous strain rates, so only this guess solves a viscosity operator"}


C4_WORKLOAD = ("adjoint_c4: 201x201 linear-elastic quasi-dynamic, constant grid, aging law, steady-state initial "
               "guess, %d RK32 steps of at most 1e4 s, rootTol 1e-14; misfit L2(surface displacement) + L2(slip velocity) against a target from "
               "seeded perturbed a(z), b(z), Dc(z) at 40 depth knots each; gradient with respect to the 120 knot "
               "values, checkpoints every 50 steps")


def run_adjoint_c4(args, dist, rank, world, local):
    """Adjoint gradient of the 201 x 201 misfit workload (2000 RK32 steps,
    120 knot parameters of a, b and Dc) and its check against central
    finite differences of the forward map (h = 1e-6 relative, 10 random
    directions in knot space)."""
    import torch
    from scycle_b200.adjoint import Adjoint, knot_matrix
    from scycle_b200.configs import make_qd_problem, write_petsc_vec
    from scycle_b200.qd import QD, inspect_in
    n, M = 201, args.c4_steps
    work = tempfile.mkdtemp(prefix="scy_c4_")
    # step sizes capped at 1e4 s: the 2000 steps stay early in the
    # interseismic period (about 0.6 years), where the response to the
    # parameters is close to linear; over longer windows nucleation amplifies
    # perturbations and central differences at h = 1e-6 carry their
    # curvature
    path = make_qd_problem(work, Ny=n, Nz=n, seed=rank, state_law="agingLaw", integrator="RK32", guess_ss=1,
                           name="c4", extra={"maxDeltaT": "1e4", "rootTol": "1e-14"})
    # the profiles are the knot interpolation itself (written as inputDir/a, b,
    # Dc), so the base run and the forward map share their parameters
    f = inspect_in(path, fields=("a", "b", "Dc"))
    z = np.arange(n) / (n - 1.0) * 30.0
    depths = np.linspace(0.0, 30.0, 40)
    P = knot_matrix(z, depths)
    base_k = [np.interp(depths, z, f[k]) for k in ("a", "b", "Dc")]
    for nm, k in zip(("a", "b", "Dc"), base_k):
        write_petsc_vec(path[:-len(".in")] + "_in_" + nm, P @ k)
    # elliptic solves to 1e-14 and the friction root to 1e-14 MPa (rootTol):
    # central differences at h = 1e-6 see the forward map's solver noise
    # amplified by 1e6
    rtol = 1e-14
    run = QD.from_in(path, solve_rtol=rtol)
    run.record_attempts(True)
    run.integrate_begin_from_in()
    run.integrate_steps(M)
    dts = run.step_sizes()[:M]
    run.close()
    q = QD.from_in(path, solve_rtol=rtol)
    q.integrate_begin_from_in()
    adj = Adjoint(q, checkpoint_every=50)
    adj.set_steps(dts)
    rng = np.random.default_rng(100 + rank)
    # small perturbations: the forward map follows the base run's step sizes,
    # which a target trajectory far from it (an event at another time) would
    # not survive
    pert_k = [base_k[0] * (1 + 0.002 * rng.standard_normal(40)), base_k[1] * (1 + 0.002 * rng.standard_normal(40)),
              base_k[2] * (1 + 0.005 * rng.standard_normal(40))]
    adj.set_params(*[P @ k for k in pert_k])
    adj.forward()
    ts, tv = adj.observations()
    ws, wv = 1.0 / np.mean(ts ** 2), 1.0 / np.mean(tv ** 2)
    adj.set_targets(ts, tv, ws, wv)
    base = [P @ k for k in base_k]
    adj.set_params(*base)
    adj.forward()  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    J0 = adj.forward()
    t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter()
    J, ga, gb, gd = adj.gradient()
    t_grad = time.perf_counter() - t0
    gk = [P.T @ g for g in (ga, gb, gd)]
    h = 1e-6

    def fd_errors(blocks, seed):
        errs = []
        drng = np.random.default_rng(seed)
        for _ in range(args.c4_dirs):
            d = [k * drng.standard_normal(40) if i in blocks else np.zeros(40) for i, k in enumerate(base_k)]
            adj.set_params(*[P @ (k + h * e) for k, e in zip(base_k, d)])
            jp = adj.forward()
            adj.set_params(*[P @ (k - h * e) for k, e in zip(base_k, d)])
            jm = adj.forward()
            fd = (jp - jm) / (2 * h)
            an = sum(g @ e for g, e in zip(gk, d))
            errs.append(abs(fd - an) / max(abs(fd), abs(an), 1e-300))
        return errs

    errs = fd_errors((0, 1, 2), 7)
    errs_ab = fd_errors((0, 1), 8)
    adj.close()
    q.close()
    return {"workload": C4_WORKLOAD % M, "steps": M, "parameters": 120, "J": J, "J_forward": J0,
            "forward_s": t_fwd, "gradient_s": t_grad, "gradient_over_forward": t_grad / t_fwd,
            "fd_check": {"directions": args.c4_dirs, "h_relative": h, "max_rel_err": max(errs) if errs else None,
                         "rel_errs": errs, "max_rel_err_a_b_only": max(errs_ab) if errs_ab else None,
                         "note": "random directions in the 120 knot values; the Dc part of the gradient is small "
                                 "near the steady-state start, so directions with a Dc component see the forward "
                                 "map's round-off amplified by 1/h; directions in a and b alone are shown beside"},
            "note": "gradient time = forward + recomputation of each checkpointed segment + reverse sweep (one "
                    "transposed elliptic solve per stage); the initial state is held fixed"}


def run_ours(args, dist, rank, world, local):
    import torch
    torch.cuda.set_device(local)
    from scycle_b200 import build
    build.build(verbose=False)
    from scycle_b200 import _lib as S
    from scycle_b200.qd import QD
    L = S.lib()
    if args.c4_only:
        r = run_adjoint_c4(args, dist, rank, world, local)
        if rank == 0:
            print(json.dumps(r))
        return
    if args.c3_only:
        r = run_ensemble_c3(args, dist, rank, world, local)
        if rank == 0:
            print(json.dumps(r))
        return
    if args.batch_only:
        if rank == 0:
            print(json.dumps(run_batched(args, dist, rank, world, local)))
        else:
            run_batched(args, dist, rank, world, local)
        return
    work = tempfile.mkdtemp(prefix="scy_bench_")
    path = make_workload(work, n=args.n, seed=rank)
    prec = "mixed" if args.precision == "mixed" else "fp64"
    q = QD.from_in(path, solve_rtol=args.rtol, precision=prec, check_every=args.check_every, precond=args.precond)
    q.integrate_begin_from_in()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > 126 MB L2

    def steps(k, e2e=False, hostbuf=None):
        for _ in range(k):
            if e2e:
                S.check(L.scy_qd_set_state(q.h, S.as_dptr(hostbuf["var"]), 0))
            st = q.integrate_steps(1)
            if e2e:
                for nm, arr in (("psi", hostbuf["psi"]), ("slip", hostbuf["slip"]), ("slipVel", hostbuf["vel"])):
                    S.check(L.scy_qd_get_field(q.h, {"psi": 0, "slip": 1, "slipVel": 2}[nm], S.as_dptr(arr)))
                hostbuf["var"][:q.Nz] = hostbuf["psi"]
                hostbuf["var"][q.Nz:] = hostbuf["slip"]
            flush.zero_()
        return st

    st0 = steps(args.warmup)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = Clocks(local) if rank == 0 else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = L.scy_launch_count()
    t_sim0, n0 = st0.t, st0.d_dt_evals
    ev0.record()
    st1 = steps(args.steps)
    ev1.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = L.scy_launch_count() - launches0
    clk = clocks.stop() if clocks else None
    ms = ev0.elapsed_time(ev1)
    ms_max = _max_over_ranks(dist, ms)
    evals = st1.d_dt_evals - n0
    sim_s = st1.t - t_sim0
    total_evals = _sum_over_ranks(dist, evals)
    total_sim_years = _sum_over_ranks(dist, sim_s / YEAR)
    value = total_evals / (ms_max / 1e3)
    syph = total_sim_years / (ms_max / 3.6e6)
    solve_its = (st1.solve_its - st0.solve_its) / max(st1.solves - st0.solves, 1)

    # end to end through the C ABI with host buffers (pinned): the state goes
    # host -> device before and device -> host after every step
    Nz = q.Nz
    pin = lambda n: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    hb = {"var": pin(2 * Nz), "psi": pin(Nz), "slip": pin(Nz), "vel": pin(Nz)}
    S.check(L.scy_qd_get_field(q.h, 0, S.as_dptr(hb["psi"])))
    S.check(L.scy_qd_get_field(q.h, 1, S.as_dptr(hb["slip"])))
    hb["var"][:Nz], hb["var"][Nz:] = hb["psi"], hb["slip"]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0 = q.integrate_steps(0)
    t0 = time.perf_counter()
    ev0.record()
    e1 = steps(args.steps, e2e=True, hostbuf=hb)
    ev1.record()
    torch.cuda.synchronize()
    e_ms = _max_over_ranks(dist, ev0.elapsed_time(ev1))
    e_evals = _sum_over_ranks(dist, e1.d_dt_evals - e0.d_dt_evals)
    e2e = {"value": e_evals / (e_ms / 1e3), "unit": "stage-solves/s", "h2d_bytes_per_step": 2 * Nz * 8,
           "d2h_bytes_per_step": 3 * Nz * 8, "sim_years_per_hour": None,
           "wall_s": time.perf_counter() - t0}

    # stencil kernel timing pass (CUDA events around each launch)
    S.check(L.scy_profile_enable(1))
    steps(min(args.steps, 20))
    torch.cuda.synchronize()
    S.check(L.scy_profile_enable(0))
    pm, pl, pb = C.c_double(), C.c_longlong(), C.c_double()
    width = 8  # the CG operator applications run in FP64 in every mode
    S.check(L.scy_profile_collect(0, width, C.byref(pm), C.byref(pl), C.byref(pb)))
    achieved = (pb.value / pl.value) / (pm.value / pl.value / 1e3) / 1e9 if pl.value else None
    peaks = _peaks()
    peak = peaks.get("hbm_gbs")
    peak_src = "measured"
    if peak is None:
        peak, peak_src = 6650.0, "fallback"
    roofline = {"kernel": "stencil_kernel (fp64 operator applications on the 401x401 grid: CG matvec, residual)",
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_src,
                "traffic": None, "launch_us": (pm.value / pl.value * 1e3) if pl.value else None,
                "algorithmic_bytes_per_launch": (pb.value / pl.value) if pl.value else None,
                "note": "the fields (1.29 MB per fp64 field) are L2-resident; DRAM traffic per launch is "
                        "far below the algorithmic bytes, so this kernel is latency/L2 bound"}
    # the same steps with the fault stress from the precomputed fault response
    # (exact to the solve tolerance; Nz + 2 solves of set-up)
    resp = None
    if not args.no_response:
        q.set_mode("response")
        r0 = q.integrate_steps(1)  # builds the response matrices
        torch.cuda.synchronize()
        ev0.record()
        r1 = steps(args.steps)
        ev1.record()
        torch.cuda.synchronize()
        r_ms = _max_over_ranks(dist, ev0.elapsed_time(ev1))
        r_evals = _sum_over_ranks(dist, r1.d_dt_evals - r0.d_dt_evals)
        resp = {"value": r_evals / (r_ms / 1e3), "unit": "stage-solves/s", "ms_per_step": r_ms / args.steps,
                "sim_years_per_hour": _sum_over_ranks(dist, (r1.t - r0.t) / YEAR) / (r_ms / 3.6e6),
                "note": "fault stress from the discrete fault response (Nz+2 solves at set-up) instead of "
                        "one elliptic solve per stage; same states to the solve tolerance"}
        q.set_mode("solve")
    cycle = None
    if not args.no_cycle:
        cycle = run_cycle(args)
    c0 = None if (args.no_c0 or rank != 0) else run_c0(args)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args)
    single = {"value": value, "unit": "stage-solves/s", "ms_per_step": ms_max / args.steps,
              "sim_years_per_hour": syph, "sim_years_timed": total_sim_years, "stage_solves": total_evals,
              "cg_iterations_per_solve": solve_its, "gpu_launches": int(launches), "e2e": e2e,
              "solver": "FP64 PCG, %s preconditioner (%s), rtol %g, residual read back every %d iterations" % (
                  args.precond, "fp32" if prec == "mixed" else "fp64", args.rtol, args.check_every),
              "l2": "flushed between steps (256 MB write)", "clocks": clk, "roofline": roofline}
    q.close()
    if rank == 0 and args.n == 401:
        single["oracle_error"] = oracle_errors("c1", lambda w: make_workload(w, n=401, seed=0))
    batched = run_batched(args, dist, rank, world, local) if args.batch > 0 else None
    ensemble_c3 = run_ensemble_c3(args, dist, rank, world, local) if args.c3 > 0 else None
    adjoint_c4 = None
    if args.c4_steps > 0:
        try:
            adjoint_c4 = run_adjoint_c4(args, dist, rank, world, local)
        except Exception as e:  # reported, not fatal to the headline
            adjoint_c4 = {"error": str(e)}
    head = batched if batched else single
    if batched:
        config = batch_config(args, world)
        solver = ("FP64 CG preconditioned by fast diagonalisation (%s preconditioner; z transforms on the integer "
                  "tensor cores, banded sweeps along y), device-verified rtol %g" % (args.batch_precision, args.rtol))
        l2 = "not flushed: the ensemble's working set (about 20 MB per instance) exceeds the 126 MB L2"
    else:
        config = {"workload": WORKLOAD, "Ny": args.n, "Nz": args.n, "integrator": "RK32",
                  "parallelism": "replicas x%d" % world}
        solver, l2 = single["solver"], single["l2"]
    out = {"metric": METRIC, "value": head["value"], "unit": "stage-solves/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64 (%s preconditioner)" % ((args.batch_precision if batched else prec)),
           "data": "synthetic (seeded; reference .in format)", "config": config, "solver": solver, "l2": l2,
           "sim_years_per_hour": head["sim_years_per_hour"], "sim_years_timed": head["sim_years_timed"],
           "stage_solves": head["stage_solves"], "e2e": head["e2e"],
           "roofline": (batched.get("roofline") or roofline) if batched else roofline, "cpu_baseline": cpu,
           "gpu_launches": head["gpu_launches"], "clocks": head["clocks"],
           "batched": batched, "fp64_single": single,
           "batched_vs_fp64_single_sim_years": (batched["sim_years_per_hour"] / syph) if batched else None,
           "response_mode": resp, "cycle": cycle, "ensemble_c3": ensemble_c3, "adjoint_c4": adjoint_c4,
           "config0": c0, "v_rel_err_vs_fp64_oracle": (batched or {}).get("v_rel_err_vs_fp64_oracle")}
    if rank == 0:
        print(json.dumps(out))


CYCLE_WORKLOAD = ("qdfd_const_801: linear-elastic quasi-dynamic / fully dynamic cycles, 801x801 SBP order 4, "
                  "constant grid over 30x30 km, cs = 3.464 km/s, aging law, RK43 (PID, tol 1e-7) in the "
                  "quasi-dynamic phases, CFL wave-equation step, switch at max(eta V / tau) = 1e-3, 3 full cycles "
                  "from the steady-state guess; outgoing-characteristics damping on the boundary nodes it names")


def run_cycle(args):
    """Three quasi-dynamic / fully dynamic cycles on the 801x801 grid
    (strikeSlip_linearElastic_qd_fd).  The reference's indexing of the
    outgoing-characteristics damping leaves the box without absorbing
    boundaries, and at this size its first wave phase does not end (over five
    million steps); the run therefore uses the damping on the boundary nodes
    it names (fd_ayIndexQuirk = 0).  Quasi-dynamic phases use the fault
    response (exact to the solve tolerance)."""
    import torch
    from scycle_b200.configs import make_qdfd_problem
    from scycle_b200.cycle import Cycle
    n = args.cycle_n
    work = tempfile.mkdtemp(prefix="scy_cycle_")
    path = make_qdfd_problem(work, Ny=n, Nz=n, cycles=3, years=1000.0, extra={"fd_ayIndexQuirk": "0"})
    c = Cycle.from_in(path, solve_rtol=args.rtol, precond=args.precond)
    c.set_mode(args.cycle_mode)
    t0 = time.perf_counter()
    c.begin_from_in()
    setup = time.perf_counter() - t0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = c.run(10 ** 8)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    sw = c.switches()
    events = [s["t"] / YEAR for s in sw if s["to"] == "fd"]
    wave_us, fault_us, step_us = c.time_kernels(50)
    N = n * n
    peak = _peaks().get("hbm_gbs", 6650.0)
    wave_gbs = 24.0 * N / (wave_us * 1e-6) / 1e9
    out = {"workload": CYCLE_WORKLOAD, "Ny": n, "Nz": n, "qd_mode": args.cycle_mode, "done": int(st.done),
           "cycles": st.cycle_count, "wall_s": wall, "setup_s": setup, "sim_years": st.t / YEAR,
           "sim_years_per_hour": (st.t / YEAR) / (wall / 3600.0), "event_years": events,
           "recurrence_years": [b - a for a, b in zip(events, events[1:])],
           "steps": st.step_count, "qd_steps": st.qd_steps, "fd_steps": st.fd_steps,
           "qd_phase_s": st.qd_ms / 1e3, "fd_phase_s": st.fd_ms / 1e3,
           "fd_steps_per_s": st.fd_steps / (st.fd_ms / 1e3) if st.fd_ms else None,
           "stage_evals": st.d_dt_evals, "elliptic_solves": st.solves, "dt_fd": st.dt_fd,
           "wave_step": {"fused_us_per_step": step_us, "algorithmic_bytes_per_step": 24.0 * N,
                         "achieved_GBps": 24.0 * N / (step_us * 1e-6) / 1e9,
                         "frac_of_measured_hbm": 24.0 * N / (step_us * 1e-6) / 1e9 / peak,
                         "two_launch_form_us": {"wave_stencil": wave_us, "fault_update": fault_us,
                                                "wave_stencil_GBps": wave_gbs},
                         "note": "u, uPrev read and uNext written per node; the 15 MB working set is "
                                 "L2-resident; the fused launch overlaps the fault update (serial FP64 root "
                                 "finds on the fault row's tiles) with the body update"}}
    c.close()
    return out


def run_wave_only(args):
    """The cycle workload on an n x n grid run into its first fully dynamic
    phase, then the wave-equation and fault launches timed alone (for
    profiling)."""
    import torch
    from scycle_b200 import build
    build.build(verbose=False)
    from scycle_b200.configs import make_qdfd_problem
    from scycle_b200.cycle import Cycle
    n = args.profile_wave
    work = tempfile.mkdtemp(prefix="scy_wave_")
    path = make_qdfd_problem(work, Ny=n, Nz=n, cycles=3, years=1000.0, extra={"fd_ayIndexQuirk": "0"})
    c = Cycle.from_in(path, solve_rtol=args.rtol)
    c.set_mode("response")
    c.begin_from_in()
    st = c.run(50)
    while st.phase != 1 and not st.done:
        st = c.run(50)
    st = c.run(20)
    w, f, t = c.time_kernels(args.profile_reps)
    print(json.dumps({"wave_only": True, "n": n, "step": st.step_count, "phase": st.phase, "wave_us": w,
                      "fault_us": f, "fused_step_us": t, "wave_algorithmic_GBps": 24.0 * n * n / (w * 1e-6) / 1e9,
                      "fused_algorithmic_GBps": 24.0 * n * n / (t * 1e-6) / 1e9}))
    c.close()


def run_batch_only_profile(args):
    """The batched ensemble (args.profile_batch instances of the n x n
    workload) set up and advanced args.profile_reps steps with its launches
    issued directly (no graph), for ncu captures of its kernels."""
    import torch
    from scycle_b200 import build
    build.build(verbose=False)
    from scycle_b200.batch import Batch
    K = args.profile_batch
    work = tempfile.mkdtemp(prefix="scy_pbatch_")
    paths = [make_workload(os.path.join(work, "i%d" % s), n=args.n, seed=s) for s in range(K)]
    b = Batch(paths, solve_rtol=args.rtol, precision=args.batch_precision, transform_planes=args.transform_planes)
    b.set_graphs(False)
    b.run(args.profile_reps)
    torch.cuda.synchronize()
    print(json.dumps({"batch_only_profile": True, "instances": K, "n": args.n, "steps": args.profile_reps,
                      "autotune": b.tuning(0)}))
    b.close()


def run_stencil_only(args):
    """A x on an n x n grid (FP64, constant grid, Dirichlet/Neumann SATs): the
    operator kernel alone, sized past L2 when n >= 4097, for profiling."""
    import torch
    from scycle_b200 import build
    build.build(verbose=False)
    from scycle_b200.sbp import SbpOps
    from scycle_b200 import _lib as S
    n = args.profile_stencil
    sbp = SbpOps(4, n, n, 30.0, 30.0, np.full(n * n, 32.04))
    x = torch.randn(n * n, dtype=torch.float64, device="cuda")
    out = torch.empty_like(x)
    L = S.lib()
    for _ in range(3):
        S.check(L.scy_sbp_apply(sbp.h, 0, C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr())))
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    ev0.record()
    for _ in range(reps):
        S.check(L.scy_sbp_apply(sbp.h, 0, C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr())))
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / reps
    # x read and A x written: mu is constant and the grid separable, so the
    # operator's coefficients are 1D tables (no per-node coefficient field)
    algo = 2 * 8 * n * n
    peak = _peaks().get("hbm_gbs", 6650.0)
    print(json.dumps({"stencil_only": True, "n": n, "us_per_apply": ms * 1e3, "algorithmic_bytes": algo,
                      "algorithmic_GBps": algo / (ms / 1e3) / 1e9, "frac_of_measured_hbm": algo / (ms / 1e3) / 1e9 / peak}))


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (SciPy SuperLU direct solve + the restated fault
# and RK32) on the host's own cores.  One single-threaded oracle instance per
# core (the GPU side is an ensemble too), each with its own seed; the
# factorisations and the steady-state initial guess happen before a barrier,
# the timed steps after it.


def _host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


def _avail_bytes():
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except Exception:
        pass
    return None


_POOL_BARRIER = None


def _pool_init(barrier):
    global _POOL_BARRIER
    _POOL_BARRIER = barrier


def _oracle_worker(job):
    """One oracle instance: set-up, wait at the barrier, run ``warm`` untimed
    and then ``steps`` timed RK32 steps in one integration (the step control
    carries on from the warm-up).  The timed window starts when the oracle's
    time monitor reports step ``warm``.  Returns (timed stage-solves, timed
    seconds, timed simulated seconds, set-up seconds)."""
    import tempfile as _tf
    from oracle.problem import build_qd_problem
    from oracle.qd import QDLinearElastic
    kind, seed, n, steps, warm = job
    t0 = time.perf_counter()
    work = _tf.mkdtemp(prefix="scy_cpu_")
    if kind == "c1":
        path = make_workload(work, n=n, seed=seed)
    else:
        from scycle_b200.configs import aging_const_101
        path = aging_const_101(work, seed=seed)
    P = build_qd_problem(open(path).read())
    ora = QDLinearElastic(P, keep_history=False)
    var0 = ora.initiate_integrand()
    setup = time.perf_counter() - t0
    calls = [0]
    mark = {}
    d_dt, monitor = ora.d_dt, ora.time_monitor

    def counted_d_dt(t, var):
        calls[0] += 1
        return d_dt(t, var)

    def marked_monitor(t, dt, step):
        if step == warm and not mark:
            mark.update(t=time.perf_counter(), calls=calls[0], sim=t)
        return monitor(t, dt, step)

    ora.d_dt, ora.time_monitor = counted_d_dt, marked_monitor
    if _POOL_BARRIER is not None:
        _POOL_BARRIER.wait()
    rk = ora.integrate(max_steps=warm + steps, var0=var0)
    t1 = time.perf_counter()
    if not mark:  # the run ended inside the warm-up: nothing timed
        return 0, 1e-30, 0.0, setup
    return calls[0] - mark["calls"], t1 - mark["t"], rk.currT - mark["sim"], setup


def oracle_on_all_cores(kind, steps, n=401, max_workers=None, instances=None, warm=0):
    """Runs oracle instances of the workload on the host cores, one single-
    threaded instance per usable core at a time (capped by host memory: a
    401^2 instance holds about 4 GB at its peak), and returns the aggregate
    stage-solves/s over the timed steps.  ``instances``: how many instances
    (seeds 0 .. instances-1) to run in all, in rounds of one per core (the
    aggregate is the timed stage-solves of every round over the sum of the
    rounds' slowest timed windows); default one per core."""
    import multiprocessing as mp
    cores = _host_cores()
    per = 5e9 if kind == "c1" else 0.5e9
    avail = _avail_bytes()
    workers = cores if avail is None else max(1, min(cores, int(avail // per)))
    if max_workers:
        workers = min(workers, max_workers)
    total = instances if instances else workers
    saved = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")}
    for k in saved:
        os.environ[k] = "1"
    res, rounds, wall = [], 0, 0.0
    try:
        ctx = mp.get_context("spawn")  # the parent may already hold a CUDA context
        for first in range(0, total, workers):
            seeds = list(range(first, min(total, first + workers)))
            barrier = ctx.Barrier(len(seeds))
            with ctx.Pool(len(seeds), initializer=_pool_init, initargs=(barrier,)) as pool:
                got = pool.map(_oracle_worker, [(kind, s, n, steps, warm) for s in seeds])
            res += got
            rounds += 1
            wall += max(r[1] for r in got)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    evals = sum(r[0] for r in res)
    value = evals / wall
    return {"value": value, "unit": "stage-solves/s", "cores": workers, "host_cores": cores,
            "cpu_model": _cpu_model(), "workers": workers, "instances": total, "rounds": rounds,
            "warmup_steps_per_instance": warm, "steps_per_worker": steps, "stage_solves": evals,
            "timed_s_max": max(r[1] for r in res), "timed_s_sum_of_rounds": wall,
            "setup_s_max": max(r[3] for r in res),
            "sim_years_per_hour": sum(r[2] for r in res) / YEAR / (wall / 3600.0)}


def run_ztransform_only(args):
    """The tensor-core z transform alone at the batched ensemble's shape
    (32 instances of 401 x 401: 12832 z-lines of 401 values times a 401 x 401
    weight matrix) with the given number of digit planes, for profiling."""
    import torch
    from scycle_b200 import build
    build.build(verbose=False)
    from scycle_b200 import _lib as S
    rows, K = 32 * 401, 401
    x = torch.randn(rows, K, dtype=torch.float64, device="cuda")
    w = np.ascontiguousarray(np.random.default_rng(0).standard_normal((K, K)))
    d = torch.empty(rows, K, dtype=torch.float64, device="cuda")
    L = S.lib()
    for _ in range(args.profile_reps):
        S.check(L.scy_ozaki_matmul(C.c_void_p(x.data_ptr()), K, rows, K, S.as_dptr(w), K, K, args.profile_ztransform,
                                   C.c_void_p(d.data_ptr()), K, args.profile_ctas, args.profile_bf16))
    torch.cuda.synchronize()
    print(json.dumps({"ztransform_only": True, "rows": rows, "K": K, "planes": args.profile_ztransform,
                      "ctas_per_sm": args.profile_ctas, "bf16_digits": args.profile_bf16, "reps": args.profile_reps}))


def cpu_baseline(args):
    """The oracle on a bounded sample of the headline workload, on all host
    cores (one single-threaded instance per core)."""
    r = oracle_on_all_cores("c1", args.cpu_steps, n=args.n)
    r.update({"kind": "port",
              "sample": "%d RK32 steps of the 401x401 workload on each of %d single-threaded oracle instances "
                        "(one per core, seeds 0..%d), summed stage-solves/s; SuperLU factorisations and the "
                        "steady-state initial guess before the timed steps" % (args.cpu_steps, r["workers"],
                                                                              r["workers"] - 1)})
    return r


def run_reference(args, dist, rank, world, local):
    """The reference arm: the oracle port of the reference's CPU path timed on
    the host cores over the headline ensemble (the same ``--batch`` instances
    and seeds as one GPU's batch), each instance ``--warmup`` untimed and then
    ``--steps`` timed RK32 steps (capped by ``--cpu-steps-ref``), one single-
    threaded instance per core at a time (rank 0 only)."""
    if rank != 0:
        return
    k = max(1, min(args.steps, args.cpu_steps_ref))
    inst = args.batch if args.batch > 0 else 1
    r = oracle_on_all_cores("c1", k, n=args.n, instances=inst, warm=args.warmup)
    value = r["value"]
    cpu = dict(r)
    cpu.update({"kind": "port",
                "sample": "%d instances (seeds 0..%d) of the 401x401 workload, %d untimed and %d timed RK32 steps "
                          "each, in %d round(s) of one single-threaded oracle instance per core on %d cores; "
                          "SuperLU factorisations and the steady-state initial guess before the warm-up"
                          % (inst, inst - 1, args.warmup, k, r["rounds"], r["workers"])})
    config = batch_config(args, 1) if args.batch > 0 else {"workload": WORKLOAD, "Ny": args.n, "Nz": args.n,
                                                            "integrator": "RK32", "parallelism": "replicas x1"}
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "stage-solves/s", "n_gpus": world,
           "steps": k, "warmup": args.warmup, "ms_per_step": r["timed_s_sum_of_rounds"] * 1e3 / k,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded; reference .in format)", "config": config,
           "solver": "SciPy SuperLU direct (stands in for the reference's MUMPS Cholesky), factorised once per "
                     "instance", "host_parallelism": "one single-threaded instance per host core",
           "cpu_baseline": cpu,
           "e2e": {"value": value, "unit": "stage-solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=401)
    ap.add_argument("--precision", default="fp64", choices=["mixed", "fp64"])
    ap.add_argument("--rtol", type=float, default=1e-12)
    ap.add_argument("--check-every", type=int, default=1)
    ap.add_argument("--precond", default="auto", choices=["auto", "mg", "fd"])
    ap.add_argument("--cpu-steps", type=int, default=10, help="RK32 steps per core of the CPU baseline")
    ap.add_argument("--cpu-steps-ref", type=int, default=20, help="cap on the reference arm's timed steps per instance")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-response", action="store_true")
    ap.add_argument("--no-cycle", action="store_true", help="skip the 801x801 quasi-dynamic / fully dynamic cycles")
    ap.add_argument("--no-c0", action="store_true", help="skip the 200-year 101x101 run (config 0)")
    ap.add_argument("--batch", type=int, default=32, help="instances per GPU of the batched ensemble (0: none)")
    ap.add_argument("--batch-precision", default="fp64", choices=["fp64", "mixed", "tf32"])
    ap.add_argument("--transform-planes", type=int, default=0,
                    help="digit planes of the tensor-core z transforms (0: by precision)")
    ap.add_argument("--batch-only", action="store_true", help="measure the batched ensemble alone")
    ap.add_argument("--c3", type=int, default=128, help="instances of the power-law ensemble (0: skip)")
    ap.add_argument("--c3-only", action="store_true", help="measure the power-law ensemble alone")
    ap.add_argument("--c3-steps", type=int, default=50, help="timed steps of the power-law ensemble")
    ap.add_argument("--no-pl-ss", action="store_true",
                    help="skip the power-law steady-state guess at the default viscosity cap")
    ap.add_argument("--c4-steps", type=int, default=2000, help="RK32 steps of the adjoint workload (0: skip)")
    ap.add_argument("--c4-dirs", type=int, default=10, help="finite-difference directions of the adjoint check")
    ap.add_argument("--c4-only", action="store_true", help="run the adjoint workload alone")
    ap.add_argument("--cycle-n", type=int, default=801)
    ap.add_argument("--cycle-mode", default="response", choices=["response", "solve"])
    ap.add_argument("--profile-stencil", type=int, default=0,
                    help="time only the FP64 operator kernel on an n x n grid and exit")
    ap.add_argument("--profile-wave", type=int, default=0,
                    help="run the cycle workload on an n x n grid into a wave phase, time its two launches, exit")
    ap.add_argument("--profile-reps", type=int, default=20)
    ap.add_argument("--profile-batch", type=int, default=0,
                    help="set up this many instances of the batched workload, advance --profile-reps steps with "
                         "direct launches (for ncu) and exit")
    ap.add_argument("--profile-bf16", type=int, default=0, choices=[0, 1],
                    help="digits in bf16 (kind::f16) instead of 8-bit integers in --profile-ztransform")
    ap.add_argument("--profile-ctas", type=int, default=1, choices=[0, 1, 2],
                    help="shape of the z-transform product in --profile-ztransform: CTAs per SM (2: S <= 5), "
                         "0 the persistent shape (S <= 5)")
    ap.add_argument("--profile-ztransform", type=int, default=0,
                    help="run only the tensor-core z transform with this many digit planes (for ncu) and exit")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.profile_stencil:
        run_stencil_only(args)
        return
    if args.profile_wave:
        run_wave_only(args)
        return
    if args.profile_ztransform:
        run_ztransform_only(args)
        return
    if args.profile_batch:
        run_batch_only_profile(args)
        return
    if args.impl == "reference":
        # rank 0 alone runs the CPU reference; with no process group the other
        # ranks exit at once instead of waiting minutes at a collective
        run_reference(args, None, int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), 0)
        return
    dist, rank, world, local = _dist()
    try:
        run_ours(args, dist, rank, world, local)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
