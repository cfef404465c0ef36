#!/usr/bin/env python
"""Benchmark of the PHG assembly + Jacobi-PCG hot path on B200.

Workload (one "step"): P2 Poisson on the unit cube split into 64^3 subcubes
x 6 Kuhn tetrahedra (1,572,864 elements, 129^3 = 2,146,689 DOFs), kappa = 1,
f = 3 pi^2 sin(pi x) sin(pi y) sin(pi z), homogeneous Dirichlet BC on all
faces; element assembly into CSR (order-2 stiffness rule, order-4 RHS rule),
boundary elimination, then Jacobi-PCG from x = 0 to relative residual 1e-8.
Inputs are synthetic (generated here), not a dataset.

Metric: time to tolerance of one step in ms (lower is better), with the
mixed-precision solver (FP32 inner PCG, FP64 reliable updates; the FP64
residual meets the tolerance); the plain FP64 step is timed beside it.
  value  inputs already resident in HBM (mesh, element->DOF map, Dirichlet
         flags, f): SetMesh + SetDofMap + BuildLinearSystem + SolverPCGMixed.
  e2e    the same calls with HOST (pinned) input buffers: the host->device
         copies of the inputs and the device->host copy of the solution are
         inside the timed region.
The dominant kernel is the CSR SpMV inside PCG; its roofline is reported
against the measured HBM copy bandwidth.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 (launched by torch.distributed.run, one process per GPU)
every rank solves its own copy of the problem (replicas: the path runs on
one GPU), value = max over ranks of the step time.  --impl reference times
the reference's own CPU build (oracle/_ref/phg_dump_omp, all host threads)
on the same workload.
"""
import argparse
import gc
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

METRIC = "P2 Poisson assembly+PCG time to 1e-8 rel. resid (64^3 Kuhn cube, 2.15M DOF), 1 B200"
REF_DUMP_OMP = os.path.join(ROOT, "oracle", "_ref", "phg_dump_omp")
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--m", type=int, default=64, help=argparse.SUPPRESS)
    ap.add_argument("--no-cpu-baseline", action="store_true", help=argparse.SUPPRESS)
    # fix the SpMV layouts instead of autotuning them (profiler runs, whose
    # serialised launches make the autotuner's timings meaningless):
    # "sell:4" for the FP64 plan, "q16:2" for the mixed solver's FP32 product
    ap.add_argument("--fp64-plan", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--fp32-plan", default=None, help=argparse.SUPPRESS)
    return ap.parse_args()


def workload(m):
    return {"workload": "P2 Poisson, %d^3 subcubes x 6 Kuhn tets, kappa=1, sine RHS, "
                        "Dirichlet 0, Jacobi-PCG to rtol 1e-8 (btol=atol=0) from x=0" % m,
            "elements": 6 * m ** 3, "dofs": (2 * m + 1) ** 3, "order": 2, "rtol": 1e-8,
            "l2_flush": "inputs and CSR exceed the 126 MB L2"}


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, val in zip(names, parts[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(path))["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def committed_traffic(kernel_key):
    """dram bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/traffic.json), or None."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))[kernel_key]
    except (OSError, KeyError, ValueError):
        return None


# ---------------------------------------------------------------------------
# Replicas (--gpus N): every rank solves its own copy; the job's time is the
# slowest rank's.  The process group is only used for these two calls.
def replica_barrier(dist):
    if dist is not None and dist.is_initialized():
        dist.barrier()


def replica_max(val, dist, device=None):
    """Max of a float over all ranks (the value itself without a group)."""
    if dist is None or not dist.is_initialized():
        return val
    import torch
    t = torch.tensor([float(val)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
def write_mesh(m, path):
    from phg_b200.mesh import kuhn_cube, write_medit
    v, e = kuhn_cube(m)
    write_medit(path, v, e)


def run_reference(args, m, reps, sample_maxit, threads=None, maxit=100000):
    """Runs the reference's OpenMP build on the workload (element loop on all
    threads as examples/poisson.c does, PHG's OpenMP SpMV and BLAS-1);
    returns the JSON lines of its repetitions (rep 0 runs to tolerance or
    `maxit`, later reps stop after `sample_maxit` PCG iterations)."""
    if not os.path.exists(REF_DUMP_OMP):
        raise RuntimeError("reference build missing (oracle/_ref/phg_dump_omp)")
    with tempfile.TemporaryDirectory() as d:
        mesh = os.path.join(d, "cube.mesh")
        write_mesh(m, mesh)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads or os.cpu_count()), OMP_PROC_BIND="false")
        cmd = [REF_DUMP_OMP, "-mesh_file", mesh, "-dof_type", "P2", "-solver", "pcg",
               "-pcg_pc_type", "jacobi", "-solver_rtol", "1e-8", "-solver_btol", "0",
               "-solver_atol", "0", "-solver_maxit", str(maxit), "-map_reorder", "no",
               "-repeat", str(reps), "-sample_maxit", str(sample_maxit)]
        out = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=3600, check=True)
    return [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]


def stage_split(rec, nits_full):
    """Stage times (ms) of one reference repetition; a capped solve is
    scaled to the full iteration count."""
    return {"t_build_ms": round(1e3 * rec["t_build"], 1), "t_assemble_ms": round(1e3 * rec["t_assemble"], 1),
            "t_solve_ms": round(1e3 * rec["t_solve"] * nits_full / max(rec["nits"], 1), 1),
            "nits": int(nits_full), "threads": int(rec["threads"])}


# iterations of the one-thread sample of the reference (its solve time is
# scaled to the full count)
ONE_THREAD_SAMPLE_ITS = 20


def one_thread_reference(args, m, nits_full):
    """The reference on one thread: element loop and phgSolverAssemble in
    full, PCG for ONE_THREAD_SAMPLE_ITS iterations scaled to nits_full."""
    r = run_reference(args, m, 1, 0, threads=1, maxit=ONE_THREAD_SAMPLE_ITS)[0]
    st = stage_split(r, nits_full)
    st["value_ms"] = round(st["t_build_ms"] + st["t_assemble_ms"] + st["t_solve_ms"], 1)
    st["sample"] = ("1 thread: element loop + phgSolverAssemble in full, %d PCG iterations scaled to %d"
                    % (r["nits"], nits_full))
    return st


def reference_step_ms(rec, nits_full):
    """Stage times of one repetition; a capped solve is scaled to the full
    iteration count."""
    solve = rec["t_solve"] * (nits_full / max(rec["nits"], 1))
    return 1e3 * (rec["t_build"] + rec["t_assemble"] + solve)


def impl_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    m = args.m
    # every repetition is the full workload (element loop, phgSolverAssemble,
    # PCG to tolerance); the first `warmup` are discarded
    recs = run_reference(args, m, args.warmup + args.steps, 0)
    nits_full = recs[0]["nits"]
    timed = recs[-args.steps:]
    vals = [reference_step_ms(r, r["nits"]) for r in timed]
    v = statistics.mean(vals)
    threads = recs[0]["threads"]
    mean_rec = {k: statistics.mean(r[k] for r in timed) for k in ("t_build", "t_assemble", "t_solve")}
    mean_rec.update(nits=nits_full, threads=threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "ms",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(v, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload(m),
        "cpu_baseline": {"value": round(v, 3), "unit": "ms", "cores": threads, "kind": "reference",
                         "sample": "reference OpenMP build (oracle/_ref/phg_dump_omp), the full "
                                   "workload each step: element loop + phgSolverAssemble + FP64 "
                                   "PCG to 1e-8 (%d iterations); mesh import outside the timing"
                                   % nits_full,
                         "stages": stage_split(mean_rec, nits_full)},
        "e2e": {"value": round(v, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_nits": nits_full,
        "reference_full_solve_ms": round(1e3 * (recs[0]["t_build"] + recs[0]["t_assemble"] +
                                                recs[0]["t_solve"]), 1),
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
def impl_ours(args):
    import torch
    import phg_b200 as pb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    m, p = args.m, 2
    v, e = pb.kuhn_cube(m)
    e2l, bdry, nodes = pb.lagrange_dofs(v, e, p)
    f = pb.sine_source(nodes)
    ndof = len(bdry)
    host = {"verts": v, "elems": e, "e2l": e2l, "bdry": bdry, "f": f}
    pinned = {k: torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for k, a in host.items()}
    d = {k: t.to(dev) for k, t in pinned.items()}
    x_mixed = torch.zeros(ndof, dtype=torch.float64, device=dev)
    x_fp64 = torch.zeros(ndof, dtype=torch.float64, device=dev)
    x_host = torch.zeros(ndof, dtype=torch.float64).pin_memory()
    rtol = 1e-8

    stream = torch.cuda.Stream(dev)
    s = pb.Solver(local, stream.cuda_stream)

    def assemble(inp):
        s.set_mesh(inp["verts"], inp["elems"])
        s.set_dof_map(p, inp["e2l"], inp["bdry"])
        s.build_linear_system(f=inp["f"])

    phase_ev = []   # per timed mixed step: events between its phases

    def step(inp, x, mixed, record=False):
        if record:
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
            ev[0].record(stream)
            s.set_mesh(inp["verts"], inp["elems"])
            ev[1].record(stream)
            s.set_dof_map(p, inp["e2l"], inp["bdry"])
            ev[2].record(stream)
            s.build_linear_system(f=inp["f"])
            ev[3].record(stream)
            phase_ev.append(ev)
        else:
            assemble(inp)
        x.zero_()
        if mixed:
            _, nits, res, nupd = s.solve_pcg_mixed(out=x, rtol=rtol, btol=0.0, atol=0.0)
        else:
            _, nits, res = s.solve_pcg(out=x, rtol=rtol, btol=0.0, atol=0.0)
            nupd = 0
        if record:
            ev[4].record(stream)
        return nits, res, nupd

    def barrier():
        replica_barrier(dist)

    def max_over_ranks(val):
        return replica_max(val, dist, dev)

    def timed(inp, x, k, mixed, record=False):
        barrier()
        gc.collect()
        gc.disable()   # no collector pause inside the timed region
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = s.launch_count()
        with torch.cuda.stream(stream):
            a.record(stream)
            for _ in range(k):
                out = step(inp, x, mixed, record)
            b.record(stream)
        torch.cuda.synchronize()
        gc.enable()
        barrier()
        return max_over_ranks(a.elapsed_time(b) / k), out, s.launch_count() - l0

    if args.fp64_plan or args.fp32_plan:
        with torch.cuda.stream(stream):
            assemble(d)
            if args.fp64_plan:
                layout, param = args.fp64_plan.split(":")
                s.set_spmv_plan(layout, int(param))
            if args.fp32_plan:
                layout, param = args.fp32_plan.split(":")
                s.set_spmv_plan32(layout, int(param))
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step(d, x_mixed, True)
            step(d, x_fp64, False)
    clocks = ClockSampler(local)
    clocks.start()
    ms, (nits, res, nupd), launches = timed(d, x_mixed, args.steps, True, record=True)
    ms64, (nits64, res64, _), _ = timed(d, x_fp64, args.steps, False)
    clock_info = clocks.stop()

    # end to end through the C ABI with host buffers (mixed path)
    with torch.cuda.stream(stream):
        step(pinned, x_host, True)
    e2e_ms, _, _ = timed(pinned, x_host, max(1, args.steps), True)
    # inputs of the step, plus the initial guess the solver reads from x
    # (the solution comes back through the same host array)
    h2d = sum(t.numel() * t.element_size() for t in pinned.values()) + x_host.numel() * x_host.element_size()
    d2h = x_host.numel() * x_host.element_size()

    # accuracy: mixed vs FP64 solution, both vs the exact sine solution
    xm, x64 = x_mixed.cpu().numpy(), x_fp64.cpu().numpy()
    u = np.sin(np.pi * nodes[:, 0]) * np.sin(np.pi * nodes[:, 1]) * np.sin(np.pi * nodes[:, 2])
    rel_l2_vs_fp64 = float(np.linalg.norm(xm - x64) / np.linalg.norm(x64))

    # phase breakdown: the mean over the timed mixed steps (events between
    # the phases of each step; the phases add up to the step but for the
    # host's gaps between calls)
    phases = [float(np.mean([e[i].elapsed_time(e[i + 1]) for e in phase_ev])) for i in range(4)]
    # a rebuild on the same mesh and DOF map (new coefficient values): the
    # build after the one that recorded the pattern adds the contributions at
    # their recorded places; timed over 5 builds with kappa = 1 + 0.5 (elem % 3)
    kappa_dev = torch.from_numpy(1.0 + 0.5 * (np.arange(len(e)) % 3)).to(dev)
    rb = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    with torch.cuda.stream(stream):
        s.build_linear_system(kappa=kappa_dev, f=d["f"])   # records the pattern
        s.build_linear_system(kappa=kappa_dev, f=d["f"])
        rb[0].record(stream)
        for _ in range(5):
            s.build_linear_system(kappa=kappa_dev, f=d["f"])
        rb[1].record(stream)
        s.build_linear_system(f=d["f"])   # the benchmark's system again (kappa = 1)
    torch.cuda.synchronize()
    rebuild_ms = rb[0].elapsed_time(rb[1]) / 5
    n, nnz, _ = s.sizes()
    layout, param, tune = s.spmv_plan()

    # the dominant kernels, timed alone on the launching stream
    spmv32_ms = s.time_spmv(fp32=True, reps=50)
    spmv64_ms = s.time_spmv(fp32=False, reps=50)
    # algorithmic bytes of one product (CSR with int32 columns and row
    # pointers, x read once, y written once), FP32 and FP64 values
    b32 = 8 * nnz + 4 * (n + 1) + 8 * n
    b64 = 12 * nnz + 4 * (n + 1) + 16 * n
    # bytes the layouts in use actually move (the q16 layout stores 16-bit
    # column offsets: fewer bytes than the algorithmic count)
    lb32, lb64 = s.spmv_bytes(fp32=True), s.spmv_bytes(fp32=False)
    peak, peak_kind = measured_hbm_peak()
    ach32 = b32 / (spmv32_ms * 1e-3) / 1e9
    ach64 = b64 / (spmv64_ms * 1e-3) / 1e9

    line = {
        "metric": METRIC, "value": round(ms, 3), "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
        "data": "synthetic", "config": workload(m),
        "parallelism": "replicas x%d" % world, "path": "mixed: FP32 inner PCG, FP64 reliable updates",
        "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "kernel": "FP32 SpMV (%s layout, unroll %d)" % (tune.get("fp32_layout"), tune.get("fp32_unroll", 0)),
                     "achieved": round(ach32, 1), "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(ach32 / peak, 4), "traffic": committed_traffic("spmv32_p2_m64") if m == 64 else None,
                     "algorithmic_bytes": int(b32), "launch_ms": round(spmv32_ms, 5),
                     "layout_bytes": int(lb32),
                     "layout_gbs": round(lb32 / (spmv32_ms * 1e-3) / 1e9, 1),
                     "layout_frac": round(lb32 / (spmv32_ms * 1e-3) / 1e9 / peak, 4),
                     "note": "achieved = algorithmic (int32-CSR) bytes / time; the q16 layout moves "
                             "layout_bytes (16-bit column offsets), so achieved can exceed the copy peak"},
        "fp64": {"ms": round(ms64, 3), "mixed_over_fp64": round(ms / ms64, 4), "nits": int(nits64),
                 "spmv_ms": round(spmv64_ms, 5), "spmv_gbs": round(ach64, 1),
                 "spmv_frac": round(ach64 / peak, 4), "traffic": committed_traffic("spmv64_p2_m64") if m == 64 else None,
                 "layout_bytes": int(lb64)},
        "gpu_launches": int(launches),
        "clocks": clock_info,
        "pcg": {"nits": int(nits), "reliable_updates": int(nupd), "residual_fp64": res,
                "rel_l2_vs_fp64_solution": rel_l2_vs_fp64,
                "max_err_vs_exact": float(np.max(np.abs(xm - u))),
                "fp64_max_err_vs_exact": float(np.max(np.abs(x64 - u)))},
        "phases_ms": {"set_mesh": round(phases[0], 3), "set_dof_map": round(phases[1], 3),
                      "assemble": round(phases[2], 3), "pcg_mixed": round(phases[3], 3)},
        "assembly_melem_s": round(6 * m ** 3 / (phases[2] * 1e-3) / 1e6, 1),
        "assembly_rebuild_ms": round(rebuild_ms, 3),
        "assembly_rebuild_melem_s": round(6 * m ** 3 / (rebuild_ms * 1e-3) / 1e6, 1),
        "spmv_autotune_ms": {k: (round(v, 5) if isinstance(v, float) else v) for k, v in tune.items()},
        "n": int(n), "nnz": int(nnz),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_leg(args, m)
        # the FP64 oracle PCG (the reference's recurrence restated
        # on the CPU) on this matrix, which the parity tests show is the
        # oracle's own bit for bit; the mixed solution's distance to it
        line["pcg"].update(oracle_check(s, xm))
    s.close()
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def cpu_baseline_leg(args, m):
    """The reference's OpenMP build on all host threads (the full workload
    once) and the one-thread sample, with the stage split."""
    try:
        r0 = run_reference(args, m, 1, 0)[0]
        out = {"value": round(reference_step_ms(r0, r0["nits"]), 1), "unit": "ms",
               "cores": r0["threads"], "kind": "reference",
               "sample": "the full workload once: reference OpenMP build (oracle/_ref/phg_dump_omp), "
                         "element loop (OpenMP, as examples/poisson.c) + phgSolverAssemble + FP64 PCG "
                         "(%d its)" % r0["nits"],
               "stages": stage_split(r0, r0["nits"])}
        out["one_thread"] = one_thread_reference(args, m, r0["nits"])
        return out
    except Exception as ex:  # report, never fail the GPU measurement
        return {"value": None, "unit": "ms", "cores": os.cpu_count(), "kind": "reference",
                "sample": "failed: %s" % ex}


def oracle_check(s, xm):
    """Relative L2 distance of the mixed solution to the FP64 oracle PCG
    solution of the same system (test infrastructure, run as a comparison)."""
    try:
        from oracle import pho
        ptr, cols, vals = s.get_matrix()
        xo, no, _, _ = pho.pcg(ptr, cols, vals, s.get_diagonal(), s.get_rhs(), rtol=1e-8, btol=0.0,
                               atol=0.0)
        return {"rel_l2_vs_oracle": float(np.linalg.norm(xm - xo) / np.linalg.norm(xo)),
                "oracle_nits": int(no)}
    except Exception as ex:  # report, never fail the GPU measurement
        return {"rel_l2_vs_oracle": None, "oracle_check": "failed: %s" % ex}


def main():
    args = parse_args()
    if args.impl == "reference":
        impl_reference(args)
    else:
        impl_ours(args)


if __name__ == "__main__":
    main()
