#!/usr/bin/env python
"""Benchmark of the B200 ParMooN CD3D hot path.

Workload (one "step"): the convection-dominated CD3D problem with SUPG on
Q2 hexahedra, 64^3 cells (2,146,689 dofs, 130,422,149 nnz on the finest of 5
levels), eps = 1e-6, b = (1, 0.5, 0.25), c = 0, f = 1, u = 1 on x = 0 and
u = 0 on the rest of the boundary, Gauss3 quadrature: assembly of all five
levels (TSystemCD3D::Assemble) followed by FGMRES(40) preconditioned by one
V-cycle SSOR(2,2) with a dense coarsest solve, run until the FP64 true
residual satisfies |r| <= 1e-10 |r0| (TSystemCD3D::Solve).

  value      device time of one step (assembly + solve), seconds, inputs
             resident in HBM, FP32-stored V-cycle inside FP64 FGMRES
  e2e        the same step through the C ABI with host buffers: start
             vector and rhs copied in, solution copied out, inside the timer
  extras     finest-level assembly Mnnz/s, plain FP64-GMG time, iterations,
             FP64 residual, roofline of the dominant kernel (the FP32 SSOR
             sweep of the finest level) and of the assembly kernel, and the
             errors of the FP32-V-cycle and FP64 solutions against an
             FP64-everywhere solve of the same system to 1e-14
  cpu_baseline  the compiled reference, one sequential process, one step of
             the same workload (unscaled), timed after the GPU work

--impl reference: the compiled reference on the same workload, one
sequential process per host thread (up to --steps processes, bounded by host
memory), all timed steps running at once; value = wall time of the timed
block / steps (the host's throughput), latency per step reported beside it.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
For N > 1 (torchrun) every rank solves its own copy (replicas, weak scaling;
the problem has no exchange step on one GPU), timing is the max over ranks.
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Time to 1e-10 FP64 residual & assembly Mnnz/s: learned/FP32 MG vs FP64 MG, 1 B200"
N_CELLS, N_LEVELS = 64, 5
EPS, B, F = 1e-6, (1.0, 0.5, 0.25), 1.0
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "pmg_ref")
# FGMRES restart length of both arms: no restart occurs inside the solve to
# 1e-10 in either (19 iterations here, 25 in the reference), so both stop on
# |r| <= 1e-10 |r0| of the first residual (the reference's restart rule,
# FgmresIte.C:546-566, would otherwise re-base r0 at iteration 20)
RESTART = 40
N_FULL = (2 * N_CELLS + 1) ** 3
# DRAM traffic of one FP32 SSOR step per algorithmic byte, measured with ncu
# (dram__bytes_read.sum + dram__bytes_write.sum over the 54 colour launches of
# one step on the finest level of the 48^3 Q2 hierarchy: 0.858 GB for 0.663 GB
# algorithmic -- FP32 values, 16-bit column deltas, slice pointers, lane rows,
# vectors); the step's traffic scales with the rows and entries it sweeps
SSOR_TRAFFIC_PER_BYTE = 0.857810 / 0.662910


def pinned_f64(n):
    """A page-locked float64 host array of n entries (as numpy)."""
    import torch
    return torch.empty(n, dtype=torch.float64).pin_memory().numpy()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            P = json.load(f)
        return float(P.get("hbm_gbs", 6650.0)), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms.  The sampler
    starts before the warm-up (nvidia-smi takes a moment to begin) and only the
    samples whose timestamps fall inside the marked timed window are kept."""

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None
        self.window = None

    def __enter__(self):
        q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        import datetime
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 8:
                try:
                    ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                except ValueError:
                    continue
                self.rows.append([ts] + parts[1:])

    def mark(self, t0, t1):
        """The timed window, in time.time() seconds."""
        self.window = (t0, t1)

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.1)  # let the sample that closes the window arrive
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = self.rows
        if self.window is not None:
            t0, t1 = self.window
            rows = [r for r in rows if t0 - 0.025 <= r[0] <= t1 + 0.025]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[4 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "interval_ms": 50}


def max_over_ranks(value, dist, device=None):
    """The largest of the ranks' values (the job's time is its slowest rank's);
    the value itself without a process group."""
    if dist is None or not dist.is_initialized():
        return value
    import torch
    dev = device or ("cuda" if dist.get_backend() == "nccl" else "cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dirichlet(x, y, z):
    return (np.abs(x) < 1e-12).astype(float)


def setup(P, precision):
    levels = P.struct_hierarchy(P.Q2_HEX, N_CELLS, N_LEVELS)
    h = P.Handle(N_LEVELS, P.default_params(precision=precision, restart=RESTART))
    h.set_coefficients(P.coeff(kind=P.COEF_CONST, eps=EPS, b=B, f=F))
    P.load_hierarchy(h, levels, dirichlet=dirichlet)
    return h, levels


def ref_options():
    """pmg_ref options of the benchmarked workload (the same problem, hierarchy,
    quadrature and solver settings as this arm): Q2 SUPG 64^3 over 5 levels."""
    return dict(order=2, levels=N_LEVELS, coarse_steps=2, problem="cdsupg", eps=EPS, b1=B[0], b2=B[1], b3=B[2],
                red=1e-10, restart=RESTART, dump=0, transfer=0)


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def host_cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def mem_available():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except Exception:
        pass
    return 0


# host memory of one reference process at 64^3 / 5 levels (measured peak RSS 2.83 GB) with headroom
REF_BYTES_PER_PROCESS = 3.5e9


def run_reference(n_steps, n_warm, max_procs=None, timeout=3000):
    """The compiled reference (oracle/_ref/pmg_ref: the reference's own
    TSquareStructure3D, TAssembleMat3D, TMultiGrid3D and TFgmresIte) on the
    benchmarked workload, unscaled.  The reference is sequential, so the host's
    cores run independent copies: P processes build the hierarchy (untimed),
    do their share of the n_warm warm-up steps, wait for a common start
    signal, then do their share of the n_steps timed steps (Assemble() of all
    levels + Solve() from the zero start vector, bracketed as
    CD3D_ParMooN.C:418-463 brackets them).  Returns the per-step times, the
    wall time of the timed block (start signal to the last process's end) and
    the process count."""
    cores = host_cores()
    procs_cap = max(1, min(cores, int(mem_available() // REF_BYTES_PER_PROCESS) or 1))
    P = max(1, min(n_steps, procs_cap if max_procs is None else min(max_procs, procs_cap)))
    reps = [n_steps // P + (1 if j < n_steps % P else 0) for j in range(P)]
    warms = [n_warm // P + (1 if j < n_warm % P else 0) for j in range(P)]
    td = tempfile.mkdtemp(prefix="pmg_ref_")
    go = os.path.join(td, "go")
    workers = []
    for j in range(P):
        out = os.path.join(td, f"w{j}")
        opt = dict(ref_options(), repeat=reps[j], warmup=warms[j], start_file=go)
        cmd = [REF_BIN, "cd3d", out] + [f"{k}={v}" for k, v in opt.items()]
        workers.append((subprocess.Popen(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL), out))

    def meta(out):
        m = {}
        try:
            with open(os.path.join(out, "meta.txt")) as f:
                for line in f:
                    k, kind, v = line.split()
                    if kind == "scalar":
                        m[k] = float(v)
        except (FileNotFoundError, ValueError):
            pass
        return m

    t_end = time.time() + timeout
    while time.time() < t_end:  # every process ready (hierarchy built, warm-up done)
        if any(p.poll() not in (None, 0) for p, _ in workers):
            raise RuntimeError("a reference process failed before the timed block")
        if all("ready_epoch" in meta(o) for _, o in workers):
            break
        time.sleep(0.2)
    else:
        for p, _ in workers:
            p.kill()
        raise RuntimeError("reference processes not ready in time")
    t_go = time.time()
    open(go, "w").close()
    for p, _ in workers:
        p.wait(timeout=max(1.0, t_end - time.time()))
        if p.returncode != 0:
            raise RuntimeError(f"reference process exited with {p.returncode}")
    steps = []
    t_last = t_go
    for _, o in workers:
        m = meta(o)
        t_last = max(t_last, m["timed_end_epoch"])
        k = 0
        while f"R{k}_t_solve" in m:
            steps.append(dict(t_assemble=m[f"R{k}_t_assemble"], t_solve=m[f"R{k}_t_solve"],
                              iterations=m[f"R{k}_iterations"], rel_res=m[f"R{k}_rel_res"]))
            k += 1
    shutil.rmtree(td, ignore_errors=True)
    return dict(steps=steps, wall=t_last - t_go, procs=P, cores=cores, reps=reps)


def ref_desc(P, cores):
    return (f"reference ParMooN compiled from its sources (oracle/_ref/pmg_ref, g++ -O3 -march=native, sequential "
            f"build) on the benchmarked workload itself (Q2 SUPG 64^3, 5 levels, FGMRES({RESTART}) + V-cycle "
            f"SSOR(2,2) to 1e-10, no scaling): {P} concurrent independent processes on the host's {cores} "
            f"threads ({host_cpu_model()}); per step Assemble() of all levels + Solve() wall time")


def bench_reference(args, rank, world):
    if rank != 0:
        return
    if not os.path.exists(REF_BIN):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/pmg_ref not built (make -C oracle/ref)"}))
        return
    r = run_reference(args.steps, args.warmup)
    per = [s["t_assemble"] + s["t_solve"] for s in r["steps"]]
    value = r["wall"] / args.steps  # throughput of the whole host: seconds per solved system
    line = {"metric": METRIC, "value": value, "unit": "s", "impl": "reference", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"CD3D SUPG Q2 hexahedra {N_CELLS}^3 ({N_LEVELS} levels), eps=1e-6, b=(1,.5,.25), "
                                   f"f=1, FGMRES({RESTART}) + V-cycle SSOR(2,2), to 1e-10",
                       "n_dofs": N_FULL, "levels": N_LEVELS,
                       "parallelism": f"{r['procs']} concurrent sequential processes"},
            "value_kind": "host throughput: wall time of the timed block / steps, all processes running at once",
            "latency_s": {"median": statistics.median(per), "min": min(per), "max": max(per)},
            "assembly_s_median": statistics.median(s["t_assemble"] for s in r["steps"]),
            "solve_s_median": statistics.median(s["t_solve"] for s in r["steps"]),
            "iterations": r["steps"][0]["iterations"], "rel_res": max(s["rel_res"] for s in r["steps"]),
            "timed_wall_s": r["wall"], "processes": r["procs"], "host_threads": r["cores"],
            "host_cpu": host_cpu_model(),
            "cpu_baseline": {"value": value, "unit": "s", "cores": r["procs"], "kind": "reference",
                             "sample": ref_desc(r["procs"], r["cores"])},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def bench_ours(args, rank, world, dist):
    import ctypes
    import parmoon_b200 as P
    lib = P.lib()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    h, levels = setup(P, P.PREC_FP32)
    Fl = levels[-1]
    nnz_fine = int(Fl["rowptr"][-1])

    def sync():
        if dist is not None:
            import torch
            torch.cuda.synchronize()
            dist.barrier()

    def step():
        h.assemble(-1, P.FORM_SUPG, copy_out=False)
        t_asm, _, _ = h.timings()
        _, st, rc = h.solve()
        return t_asm + st.seconds, st, rc

    with ClockSampler(local) as clk:
        for _ in range(args.warmup):
            step()
        sync()
        cnt0 = ctypes.c_ulonglong()
        lib.pmg_launch_count(ctypes.byref(cnt0))
        times, stats = [], []
        nvtx = None
        if os.environ.get("BENCH_NVTX") == "1":  # marks the timed region for profiler range filters
            import torch
            nvtx = torch.cuda.nvtx
            nvtx.range_push("timed_step")
        t_epoch = time.time()
        t_wall = time.perf_counter()
        for _ in range(args.steps):
            t, st, rc = step()
            if rc != 0:
                raise RuntimeError(f"solve failed with status {rc}")
            times.append(t)
            stats.append(st)
        t_wall = time.perf_counter() - t_wall
        clk.mark(t_epoch, time.time())
        if nvtx is not None:
            nvtx.range_pop()
    cnt1 = ctypes.c_ulonglong()
    lib.pmg_launch_count(ctypes.byref(cnt1))
    sync()
    step_time = max_over_ranks(statistics.mean(times), dist)

    # finest-level assembly throughput (one Assemble() of the finest level)
    asm_fine = []
    for _ in range(3):
        h.assemble(N_LEVELS - 1, P.FORM_SUPG, copy_out=False)
        asm_fine.append(h.timings()[0])
    t_asm_fine = min(asm_fine)

    # roofline of the dominant kernel: the FP32 SSOR step on the finest level
    hbm, peak_kind = peaks()
    sec, by, fl = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    P._check(lib.pmg_time_kernel(h.h, 3, N_LEVELS - 1, 0, 5, ctypes.byref(sec), ctypes.byref(by), ctypes.byref(fl)))
    ssor = dict(seconds=sec.value, bytes=by.value, gbs=by.value / sec.value / 1e9)
    P._check(lib.pmg_time_kernel(h.h, 1, N_LEVELS - 1, 0, 5, ctypes.byref(sec), ctypes.byref(by), ctypes.byref(fl)))
    spmv32 = dict(seconds=sec.value, bytes=by.value, gbs=by.value / sec.value / 1e9)
    P._check(lib.pmg_time_kernel(h.h, 0, N_LEVELS - 1, 0, 5, ctypes.byref(sec), ctypes.byref(by), ctypes.byref(fl)))
    spmv64 = dict(seconds=sec.value, bytes=by.value, gbs=by.value / sec.value / 1e9)
    P._check(lib.pmg_time_kernel(h.h, 4, N_LEVELS - 1, P.FORM_SUPG, 3, ctypes.byref(sec), ctypes.byref(by),
                                 ctypes.byref(fl)))
    asm = dict(seconds=sec.value, bytes=by.value, gbs=by.value / sec.value / 1e9, tflops=fl.value / sec.value / 1e12)

    # end to end through the C ABI with host buffers: the right-hand side comes
    # back to page-locked host memory, the start vector (zero) and the rhs go
    # in from it, the solution comes back into it, every step
    N = Fl["N"]
    rhs_h, sol_h = pinned_f64(N), pinned_f64(N)
    e2e_t = []
    for _ in range(max(1, min(args.steps, 3))):
        t0 = time.perf_counter()
        h.assemble(-1, P.FORM_SUPG, copy_out=False)
        h.get_rhs(N_LEVELS - 1, out=rhs_h)
        sol_h.fill(0.0)
        x, st, rc = h.solve(sol=sol_h, rhs=rhs_h, inplace=True)
        e2e_t.append(time.perf_counter() - t0)
    e2e = statistics.median(e2e_t)

    # level set-up of the finest level (TSquareStructure3D + Sort): host builder
    # (OpenMP) against the device builder (pmg_build_level_csr: pattern on the
    # device, then installed with pattern checks, row colouring and host mirror)
    import ctypes as C_
    rp_h = np.empty(N + 1, dtype=np.int32)
    ed = np.ascontiguousarray(Fl["elem_dof"], dtype=np.int32)
    t0 = time.perf_counter()
    P._check(lib.pmg_struct_csr(C_.c_int(ed.size // 27), C_.c_int(27), ed.ctypes.data_as(C_.c_void_p), C_.c_int(N),
                                C_.c_int(Fl["active_bound"]), rp_h.ctypes.data_as(C_.c_void_p), None))
    kc_h = np.empty(int(rp_h[-1]), dtype=np.int32)
    P._check(lib.pmg_struct_csr(C_.c_int(ed.size // 27), C_.c_int(27), ed.ctypes.data_as(C_.c_void_p), C_.c_int(N),
                                C_.c_int(Fl["active_bound"]), rp_h.ctypes.data_as(C_.c_void_p),
                                kc_h.ctypes.data_as(C_.c_void_p)))
    t_host_csr = time.perf_counter() - t0
    hs = P.Handle(1)
    hs.build_level_csr(0, ed, 27, N, Fl["active_bound"])  # first use: module loading, allocations
    t0 = time.perf_counter()
    hs.build_level_csr(0, ed, 27, N, Fl["active_bound"])
    t_dev_csr = time.perf_counter() - t0
    c_dev, c_inst = C_.c_double(), C_.c_double()
    P._check(lib.pmg_setup_timings(hs.h, C_.byref(c_dev), C_.byref(c_inst)))
    hs.close()

    # plain FP64 GMG on the same problem (the method the FP32 V-cycle is compared with)
    x32 = h.get_solution()
    h.set_params(P.default_params(precision=P.PREC_FP64, restart=RESTART))
    fp64 = []
    for _ in range(2):
        _, st64, rc64 = h.solve()
        fp64.append((st64.seconds, st64.iterations, st64.rel_res, rc64, st64.vcycle_seconds))
    fp64_s = min(x[0] for x in fp64)
    x64 = h.get_solution()
    # error of both 1e-10 solutions against an FP64-everywhere solve of the
    # same system to |r| <= 1e-14 |r0| (FP64 V-cycle, FP64 FGMRES)
    h.set_params(P.default_params(precision=P.PREC_FP64, restart=RESTART, lin_red=1e-14, lin_maxit=300))
    _, st_t, rc_t = h.solve()
    xt = h.get_solution()
    nt = float(np.linalg.norm(xt))
    err = {"fp32_vcycle_solve": float(np.linalg.norm(x32 - xt)) / nt,
           "fp64_gmg_solve": float(np.linalg.norm(x64 - xt)) / nt,
           "fp32_vs_fp64_solve": float(np.linalg.norm(x32 - x64)) / float(np.linalg.norm(x64)),
           "fp64_everywhere_rel_res": st_t.rel_res, "fp64_everywhere_status": rc_t,
           "note": "relative L2 errors of the 1e-10 solutions against the FP64-everywhere solve to 1e-14"}

    # the learned-smoother FP32 V-cycle in FP64 FGMRES on the same problem: the
    # stencil network on every level's Q2 node lattice ((2n+1)^3 nodes), the
    # committed weights, the SSOR guard on; the timed solve includes the
    # network's forward on every level (it runs once per assembly)
    learned = None
    if os.path.exists(WEIGHTS):
        w = np.fromfile(WEIGHTS, dtype=np.float32)
        for l, L in enumerate(levels):
            h.set_lattice(l, 2 * L["n"] + 1, L["dof_lat"])
        h.set_learned_weights(w)
        h.set_params(P.default_params(precision=P.PREC_FP32, restart=RESTART, smoother=P.SMOOTHER_LEARNED))
        h.solve()  # warm-up: graph capture
        h.set_learned_weights(w)
        _, stl, rcl = h.solve()
        xl = h.get_solution()
        learned = {"solve_s": stl.seconds, "network_and_setup_s": stl.setup_seconds, "iterations": stl.iterations,
                   "rel_res": stl.rel_res, "status": rcl,
                   "smoother_used": "learned" if stl.smoother_used == P.SMOOTHER_LEARNED else "ssor",
                   "rho_plain": stl.rho_plain, "rho_learned": stl.rho_learned, "learned_cycles": stl.learned_cycles,
                   "speedup_vs_fp64_gmg": fp64_s / stl.seconds,
                   "err_vs_fp64_everywhere": float(np.linalg.norm(xl - xt)) / nt,
                   "weights": os.path.relpath(WEIGHTS, os.path.dirname(os.path.abspath(__file__)))}

    line = None
    if rank == 0:
        cpu = None
        if os.path.exists(REF_BIN) and not args.no_cpu and world == 1:  # the CPU baseline is an N=1 figure
            # one sequential reference process, one step of the same workload
            # (after the GPU timing, so the two do not share the host)
            r = run_reference(1, 0, max_procs=1)
            s0 = r["steps"][0]
            cpu = {"value": s0["t_assemble"] + s0["t_solve"], "unit": "s", "cores": 1, "kind": "reference",
                   "sample": ref_desc(1, r["cores"]).replace("concurrent independent processes", "process")
                   + "; one step",
                   "assembly_s": s0["t_assemble"], "solve_s": s0["t_solve"], "iterations": s0["iterations"],
                   "rel_res": s0["rel_res"], "host_cpu": host_cpu_model()}
        st = stats[-1]
        line = {
            "metric": METRIC, "value": step_time, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_time * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
            "config": {"workload": f"CD3D SUPG Q2 hexahedra {N_CELLS}^3 ({N_LEVELS} levels), eps=1e-6, b=(1,.5,.25), f=1, "
                                   f"FGMRES({RESTART}) + V-cycle SSOR(2,2) FP32, dense coarse solve, to 1e-10",
                       "n_dofs": N, "nnz_fine": nnz_fine, "levels": N_LEVELS,
                       "l2": "inputs larger than L2 (finest matrix 1.04 GB FP64 values + 0.52 GB indices)",
                       "parallelism": f"replicas x{world}"},
            "iterations": st.iterations, "rel_res_fp64": st.rel_res, "res0": st.res0,
            "assembly_mnnz_s": nnz_fine / t_asm_fine / 1e6, "assembly_fine_s": t_asm_fine,
            "fp64_gmg": {"solve_s": fp64_s, "iterations": fp64[0][1], "rel_res": fp64[0][2], "status": fp64[0][3],
                         "vcycle_s": fp64[0][4]},
            "err_vs_fp64": err,
            "learned_fp32": learned,
            "setup_csr_s": {"host_builder": t_host_csr, "device_builder": c_dev.value,
                            "device_entry_total": t_dev_csr, "device_entry_install": c_inst.value,
                            "note": "finest-level CSR pattern (TSquareStructure3D + Sort), wall time; "
                                    "device_builder = the pattern on the device (upload included); the entry "
                                    "then installs it (pattern checks, greedy row colouring, host mirror)"},
            "fp32_solve_s": statistics.mean(s.seconds for s in stats),
            "fp32_solve_setup_s": statistics.mean(s.setup_seconds for s in stats),
            "fp32_vcycle_s": statistics.mean(s.vcycle_seconds for s in stats),
            "wall_s_per_step": t_wall / args.steps,
            "roofline": {"bound": "hbm", "kernel": "k_sell_gs<float,K> (FP32 multicolour SSOR step on SELL-32, finest level)",
                         "achieved": ssor["gbs"], "peak": hbm, "unit": "GB/s", "frac": ssor["gbs"] / hbm,
                         "traffic": ssor["bytes"] * SSOR_TRAFFIC_PER_BYTE,
                         "traffic_note": "ncu DRAM bytes of one SSOR step at 48^3, scaled by the algorithmic bytes", "peak_kind": peak_kind, "bytes_per_launch": ssor["bytes"],
                         "launch_s": ssor["seconds"]},
            "roofline_spmv64": {"achieved": spmv64["gbs"], "frac": spmv64["gbs"] / hbm, "bytes": spmv64["bytes"]},
            "roofline_spmv32": {"achieved": spmv32["gbs"], "frac": spmv32["gbs"] / hbm, "bytes": spmv32["bytes"]},
            "roofline_assembly": {"kernel": "k_tc_setup<Q2,27> + k_assemble_tc16<Q2> (reference-table contraction "
                                            "on the FP64 tensor cores, mma.sync m8n8k4 f64; finest level, all 8 "
                                            "element colours, matrix and rhs zeroed first)",
                                  "achieved_gbs": asm["gbs"], "frac_hbm": asm["gbs"] / hbm,
                                  "achieved_tflops_fp64": asm["tflops"], "bytes": asm["bytes"], "launch_s": asm["seconds"]},
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": 2 * N * 8, "d2h_bytes_per_step": 2 * N * 8},
            "gpu_launches": int(cnt1.value - cnt0.value),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    h.close()


def bench_dd(args, rank, world, dist):
    """--dd: the domain-decomposed solve (pmg_solve_dd) of the same problem over
    the ranks (z-slabs, one GPU per rank, NCCL halo exchange and sums): one step
    = assembly of every level of the rank's subdomain + the solve to 1e-10;
    value = the slowest rank's mean step time (strong scaling: the problem is
    the same at every rank count).  The slab count must divide the coarsest
    level's cells per direction."""
    import torch
    import parmoon_b200 as P
    from parmoon_b200 import dd
    glob, loc = dd.local_hierarchy(P.Q2_HEX, N_CELLS, N_LEVELS, world, rank)
    h = P.Handle(N_LEVELS, P.default_params(precision=P.PREC_FP32, restart=RESTART))
    h.set_coefficients(P.coeff(kind=P.COEF_CONST, eps=EPS, b=B, f=F))
    dd.load_subdomain(h, loc, dirichlet=dirichlet)
    comm = dd.TorchComm(dist, loc[-1])
    c = comm.struct(P.lib())
    h.set_halo(comm.send_idx, comm.recv_idx, comm.send_buf.data_ptr(), comm.recv_buf.data_ptr())

    def step():
        h.assemble(-1, P.FORM_SUPG, copy_out=False)
        t_asm = h.timings()[0]
        _, st, rc = h.solve_dd(c)
        return t_asm + st.seconds, st

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    dist.barrier()
    times = []
    for _ in range(args.steps):
        t, st = step()
        times.append(t)
    torch.cuda.synchronize()
    dist.barrier()
    value = max_over_ranks(statistics.mean(times), dist)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
                          "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
                          "scaling": "strong", "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
                          "mode": "domain-decomposed (pmg_solve_dd)",
                          "config": {"workload": f"CD3D SUPG Q2 hexahedra {N_CELLS}^3 ({N_LEVELS} levels), "
                                                 f"{world} z-slab subdomains", "parallelism": f"dd{world}"},
                          "iterations": st.iterations, "rel_res_fp64": st.rel_res}))
    h.close()


def config_line(name, extra):
    line = {"metric": METRIC, "impl": "ours", "config_name": name, "n_gpus": 1, "dtype": "f64+f32",
            "data": "synthetic", "higher_is_better": False, "unit": "s"}
    line.update(extra)
    print(json.dumps(line))


def run_config(name, steps):
    """The other workloads of the benchmark suite, one JSON line each (not the
    driver's bench line): device times of assembly and solve, FP32 V-cycle vs
    plain FP64 GMG, FP64 true residual."""
    import parmoon_b200 as P
    from parmoon_b200.configs import lognormal_modes
    if name == "poisson_q1_32":
        # Poisson Q1 32^3 (35,937 dofs), sine rhs, homogeneous Dirichlet, Gauss2, 4 levels, SSOR(2,2) FGMRES
        levels = P.struct_hierarchy(P.Q1_HEX, 32, 4)
        mk = lambda prec: P.default_params(precision=prec)
        coef = P.coeff(kind=P.COEF_SINE_RHS, eps=1.0)
        form, dirv, nl = P.FORM_GALERKIN, None, 4
    elif name == "p2tet_lognormal_64":
        # P2 tetrahedra: 64^3 hexahedra x 6 Kuhn tetrahedra (1,572,864 cells, 2,146,689 dofs), interior
        # vertices jittered by up to 0.2 h, lognormal diffusion (sigma 1, correlation 0.1), b = 0, f = 1,
        # the 5-point degree-3 tetrahedral rule the workload names
        levels = P.struct_hierarchy(P.P2_TET, 64, 5, jitter=0.2, seed=1)
        mk = lambda prec: P.default_params(precision=prec, quad_rule=P.QUAD_KEAST5)
        coef = P.coeff(kind=P.COEF_LOGNORMAL, eps=1.0, f=1.0, modes=lognormal_modes(1))
        form, dirv, nl = P.FORM_GALERKIN, None, 5
    else:
        raise ValueError(name)
    h = P.Handle(nl, mk(P.PREC_FP32))
    h.set_coefficients(coef)
    P.load_hierarchy(h, levels, dirichlet=dirv)
    out = {}
    for prec, tag in ((P.PREC_FP32, "fp32"), (P.PREC_FP64, "fp64")):
        h.set_params(mk(prec))
        ta, ts, its, rel = [], [], 0, 0.0
        for k in range(steps + 2):
            h.assemble(-1, form, copy_out=False)
            t_asm = h.timings()[0]
            _, st, rc = h.solve()
            if rc != 0:
                raise RuntimeError(f"{name}: solve status {rc}")
            if k >= 2:
                ta.append(t_asm)
                ts.append(st.seconds)
            its, rel = st.iterations, st.rel_res
        out[tag] = {"assembly_s": statistics.mean(ta), "solve_s": statistics.mean(ts), "iterations": its,
                    "rel_res_fp64": rel}
    F = levels[-1]
    config_line(name, {"value": out["fp32"]["assembly_s"] + out["fp32"]["solve_s"], "steps": steps,
                       "n_dofs": int(F["N"]), "nnz_fine": int(F["rowptr"][-1]), "levels": nl, **out})
    h.close()


def run_tcd(steps):
    """Time-dependent CD (TCD3D): Q1 128^3 (2,146,689 dofs, 5 levels), Crank-Nicolson, tau = 1e-3,
    eps = 1e-4, rotating convection b = (-(y-.5), x-.5, 0.2 sin 2 pi t), Gaussian bump (sigma 0.05 at
    (0.3, 0.5, 0.5)) as initial value, mass and SUPG stiffness reassembled on every level every step,
    FP32 V-cycle in FP64 FGMRES: device time per time step."""
    import parmoon_b200 as P
    nl, tau = 5, 1e-3
    levels = P.struct_hierarchy(P.Q1_HEX, 128, nl)
    h = P.Handle(nl, P.default_params(precision=P.PREC_FP32))
    P.load_hierarchy(h, levels)
    F = levels[-1]
    x = F["dof_xyz"]
    u = np.exp(-((x[:, 0] - 0.3) ** 2 + (x[:, 1] - 0.5) ** 2 + (x[:, 2] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u[F["active_bound"]:] = 0.0
    theta = (0.5, 0.5, 0.5, 0.5)  # Crank-Nicolson (TimeDiscRout.C: THETA1..4)
    t = 0.0
    h.set_coefficients(P.coeff(kind=P.COEF_ROTATING, eps=1e-4, f=0.0, t=t))
    h.assemble(-1, P.FORM_MASS_SUPG, copy_out=False)
    times, its, t_asm, t_sol = [], [], [], []
    for k in range(steps + 2):
        t += tau
        h.set_coefficients(P.coeff(kind=P.COEF_ROTATING, eps=1e-4, f=0.0, t=t))
        h.assemble(-1, P.FORM_MASS_SUPG, copy_out=False)
        t_m = h.timings()[0]
        h.assemble(-1, P.FORM_SUPG, copy_out=False)
        t_a = h.timings()[0]
        h.tcd_system(tau, theta, u_old=u if k == 0 else None)
        _, st, rc = h.solve()
        h.tcd_restore()
        if rc != 0:
            raise RuntimeError(f"tcd: solve status {rc}")
        if k >= 2:
            times.append(t_m + t_a + st.seconds)
            t_asm.append(t_m + t_a)
            t_sol.append(st.seconds)
            its.append(st.iterations)
    config_line("tcd_q1_128_cn", {"value": statistics.mean(times), "unit": "s per time step", "steps": steps,
                                  "n_dofs": int(F["N"]), "nnz_fine": int(F["rowptr"][-1]), "levels": nl,
                                  "iterations_mean": float(np.mean(its)),
                                  "assembly_s": statistics.mean(t_asm), "solve_s": statistics.mean(t_sol),
                                  "projected_200_steps_s": 200 * statistics.mean(times)})
    h.close()


KERNELS = {"spmv64": 0, "spmv32": 1, "ssor64": 2, "ssor32": 3, "assemble": 4, "coarse_factor": 6, "learned_fwd": 7}
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "parmoon_b200", "weights", "stencil_net_q1.f32")


def profile_kernel(name):
    """Time one kernel family on the finest level only (the command the ncu
    captures run: the first matching launches are the finest level's)."""
    import ctypes
    import parmoon_b200 as P
    lib = P.lib()
    levels = P.struct_hierarchy(P.Q2_HEX, N_CELLS, N_LEVELS)
    h = P.Handle(N_LEVELS, P.default_params(precision=P.PREC_FP32))
    h.set_coefficients(P.coeff(kind=P.COEF_CONST, eps=EPS, b=B, f=F))
    P.load_hierarchy(h, levels, dirichlet=dirichlet)
    fine = 0 if name == "coarse_factor" else N_LEVELS - 1
    if name != "assemble":
        h.assemble(fine, P.FORM_SUPG, copy_out=False)
    if name == "learned_fwd":
        # the Q2 dofs of the finest level form a (2n+1)^3 node lattice
        h.set_lattice(fine, 2 * N_CELLS + 1, levels[fine]["dof_lat"])
        h.set_learned_weights(np.fromfile(WEIGHTS, dtype=np.float32))
    sec, by, fl = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    P._check(lib.pmg_time_kernel(h.h, KERNELS[name], fine, P.FORM_SUPG, 3, ctypes.byref(sec), ctypes.byref(by),
                                 ctypes.byref(fl)))
    hbm, kind = peaks()
    print(json.dumps({"kernel": name, "n_cells": N_CELLS, "levels": N_LEVELS, "level": fine, "n_dofs": levels[fine]["N"],
                      "nnz": int(levels[fine]["rowptr"][-1]), "seconds": sec.value, "bytes": by.value,
                      "flops": fl.value, "gbs": by.value / sec.value / 1e9, "hbm_frac": by.value / sec.value / 1e9 / hbm,
                      "tflops": fl.value / sec.value / 1e12, "peak_kind": kind}))
    h.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--n-cells", type=int, default=64, help="cells per direction (64 = the benchmarked workload)")
    ap.add_argument("--levels", type=int, default=5)
    ap.add_argument("--profile-kernel", choices=sorted(KERNELS), default=None,
                    help="time one kernel on the finest level only (the profiling command)")
    ap.add_argument("--peaks", action="store_true",
                    help="print the FP64 FMA, FP64 DMMA and BF16 mma.sync throughput of this GPU")
    ap.add_argument("--dd", action="store_true",
                    help="domain-decomposed solve over the ranks (launch with torchrun, one GPU per rank)")
    ap.add_argument("--config", choices=["poisson_q1_32", "p2tet_lognormal_64", "tcd_q1_128_cn"], default=None,
                    help="run one of the other workloads instead of the bench line")
    args = ap.parse_args()
    global N_CELLS, N_LEVELS, N_FULL
    N_CELLS, N_LEVELS = args.n_cells, args.levels
    N_FULL = (2 * N_CELLS + 1) ** 3
    if args.profile_kernel:
        profile_kernel(args.profile_kernel)
        return
    if args.peaks:
        import parmoon_b200 as P
        fma, dmma, hmma = P.measure_peaks()
        print(json.dumps({"fp64_fma_tflops": fma, "fp64_dmma_tflops": dmma, "bf16_mma_sync_tflops": hmma}))
        return
    if args.config == "tcd_q1_128_cn":
        run_tcd(args.steps)
        return
    if args.config:
        run_config(args.config, args.steps)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.dd:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        bench_dd(args, rank, world, tdist)
        tdist.barrier()
        tdist.destroy_process_group()
        return
    if args.impl == "ours" and world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    elif world > 1:
        pass
    if args.impl == "reference":
        bench_reference(args, rank, world)
    else:
        bench_ours(args, rank, world, dist)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
