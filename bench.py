#!/usr/bin/env python3
"""Benchmark of the HPCG PCG path on B200.

One step = one HPCG CG set (50 preconditioned CG iterations from x = 0, tolerance
0, as the timed loop of src/main.cpp:334-340) on the 512^3 problem (134M rows,
4 MG levels, 27-point stencil, FP64), generated on the device.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line on rank 0. Under torchrun (N > 1) the ranks, one per GPU,
are the reference's MPI decomposition: each owns a 512^3 block of the
(npx*512) x (npy*512) x (npz*512) grid (process grid as the reference factors
N), exchanges halos with its neighbours over NCCL before every SpMV and
symmetric Gauss-Seidel step and allreduces every dot product, as HPCG's weak
scaling runs do ("scaling": "weak"); the value is the global problem's HPCG
flops over the slowest rank's time. --replicas instead solves N independent
512^3 problems.

value: HPCG GFLOP/s (the reference FLOP model, src/ReportResults.cpp:75-99) with
b and x resident in HBM. e2e: the same metric through the C ABI with pinned
host b and x (uploaded, solved, x downloaded every step).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "HPCG GFLOP/s & HBM GB/s at 512^3; FP32-MG vs FP64 time to 1e-9 residual"
# a level's column index as the kernels read it (hpcg_b200_level_packed): the
# "column_form" fields of the JSON line hold these codes
COLUMN_FORMS = {0: "32-bit columns", 1: "8-bit offsets", 2: "16-bit offsets",
                3: "diagonal form: 27 bases and 27 x 128 sink bits per 128-row tile"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=512, help="grid side (nx = ny = nz)")
    ap.add_argument("--iters", type=int, default=50, help="CG iterations per set")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-n", type=int, default=128, help="grid side of the CPU reference sample")
    ap.add_argument("--ref-seconds", type=float, default=20.0, help="CPU seconds budget of a reference sample")
    ap.add_argument("--no-mixed", action="store_true", help="skip the FP32 V-cycle vs FP64 time-to-1e-9 comparison")
    ap.add_argument("--mixed-rhs", default="both", choices=["hpcg", "uniform", "both"],
                    help="right-hand side(s) of the mixed-precision comparison: b = 27 - nnz, U[-1,1], or both")
    ap.add_argument("--mixed-tol", type=float, default=1e-9)
    ap.add_argument("--no-adjoint", action="store_true", help="skip the 128^3 implicit-adjoint timing")
    ap.add_argument("--no-multi", action="store_true", help="skip the 256^3, 8 right-hand-side comparison")
    ap.add_argument("--multi-n", type=int, default=256, help="grid side of the 8 right-hand-side comparison")
    ap.add_argument("--no-batch", action="store_true", help="skip the 16-problem batched comparison")
    ap.add_argument("--replicas", action="store_true",
                    help="with N > 1 GPUs: N independent problems instead of one decomposed problem")
    ap.add_argument("--decomposed", action="store_true",
                    help="run the decomposed (halo + allreduce) arm even on one GPU (a one-rank grid)")
    ap.add_argument("--vcycle", type=int, default=0, metavar="N",
                    help="one FP32 and one FP64 V-cycle of an N^3 problem, after two of each untimed, between "
                         "cudaProfilerStart and cudaProfilerStop, every kernel launched on the stream (a launch "
                         "list under ncu --profile-from-start off; the ncu summaries in profiles/)")
    ap.add_argument("--case", type=int, default=0, metavar="N",
                    help="the small profiling case instead of the bench: an N^3 problem, two V-cycles, a "
                         "3-iteration CG and a 3-iteration CG around the FP32 V-cycle, every kernel launched on "
                         "the stream (the ncu summaries in profiles/)")
    return ap.parse_args()


def profile_vcycle(n):
    """The V-cycle launch list's workload: an n^3 problem, two FP32 and two
    FP64 V-cycles untimed (the first tunes), then one of each between
    cudaProfilerStart and cudaProfilerStop, in colour order on the library's
    vectors. Prints the tuned configurations."""
    os.environ.setdefault("HPCG_B200_GRAPH", "0")
    import torch
    from hpcg_b200 import binding as B
    P = B.Problem.generate(n, n, n, 4, 0)
    r = torch.rand(n ** 3, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    x = torch.zeros_like(r)
    for _ in range(2):
        P.ComputeMG_f32(r, x)
        P.ComputeMG(r, x)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    P.ComputeMG_f32(r, x)
    P.ComputeMG(r, x)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"vcycle": n, "level_config": P.level_config_string()}))
    P.free()
    return 0


def profile_case(n):
    """The case the ncu summaries capture: a few launches of every kernel of a
    CG iteration at n^3, launched one by one on the stream (kernels inside the
    CG loop's graph cannot be captured by the profiler). Prints the tuned
    configurations and each level's column form."""
    os.environ.setdefault("HPCG_B200_GRAPH", "0")
    import torch
    from hpcg_b200 import binding as B
    P = B.Problem.generate(n, n, n, 4, 0)
    r = torch.rand(n ** 3, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    z = torch.zeros_like(r)
    for _ in range(2):
        P.ComputeMG(r, z)
    b = torch.empty_like(r)
    P.get_rhs(b)
    x = torch.zeros_like(r)
    P.CG(b, x, 3, 0.0, True)
    x.zero_()
    P.CG_mixed(b, x, 3, 0.0)
    torch.cuda.synchronize()
    print(json.dumps({"case": n, "configs": [P.level_config(l) for l in range(4)],
                      "column_forms": [P.level_pack_width(l) for l in range(4)],
                      "level_config": P.level_config_string()}))
    P.free()
    return 0


# ---------------------------------------------------------------------------
# CPU reference (the reference's own CG_ref, OpenMP build, in a subprocess)
# ---------------------------------------------------------------------------

def reference_timer_path():
    return os.path.join(HERE, "oracle", "_ref", "hpcg_ref_timer")


def run_reference_sample(n, iters, reps, warmup):
    """Times the reference's CG_ref at n^3 (all host threads). Returns the timer's JSON."""
    exe = reference_timer_path()
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    out = subprocess.run([exe, str(n), str(n), str(n), str(iters), str(reps), str(warmup)], env=env,
                         capture_output=True, text=True, timeout=1800)
    if out.returncode != 0:
        raise RuntimeError(f"reference timer failed: {out.stderr[-500:]}")
    return json.loads(out.stdout.strip().splitlines()[-1])


def reference_iters_for(n, seconds, reps):
    """Iterations per call so that reps calls take about `seconds` on this host:
    the reference runs ~1.5 GFLOP/s per core-bound MG at 128^3 (serial SYMGS)."""
    from hpcg_b200 import metrics
    per_iter = metrics.hpcg_flops(n, n, n, 1) - metrics.hpcg_flops(n, n, n, 0)
    it = int(seconds * 1.5e9 / max(per_iter, 1.0) / max(reps, 1))
    return max(1, min(50, it))


def cpu_baseline(args):
    exe = reference_timer_path()
    if os.path.exists(exe):
        iters = reference_iters_for(args.ref_n, args.ref_seconds, 1)
        r = run_reference_sample(args.ref_n, iters, 1, 0)
        return {"value": round(r["flops_per_call"] / r["mean_s"] / 1e9, 4), "unit": "GFLOP/s",
                "cores": r["threads"], "kind": "reference",
                "sample": f"CG_ref of the reference (OpenMP build, its own flags), {args.ref_n}^3, "
                          f"{iters} iterations, 1 call ({r['mean_s']:.2f} s); the reference cannot "
                          f"generate 512^3 (nnz overflows its int local_int_t)"}
    # the C restatement (serial), when the reference was not built here
    from oracle import oracle as O
    from hpcg_b200 import metrics
    n = min(args.ref_n, 64)
    P = O.generate(n)
    t0 = time.perf_counter()
    O.cg(P.levels, P.b, P.x, 10, 0.0)
    dt = time.perf_counter() - t0
    return {"value": round(metrics.hpcg_flops(n, n, n, 10) / dt / 1e9, 4), "unit": "GFLOP/s", "cores": 1,
            "kind": "port", "sample": f"C restatement of CG_ref, {n}^3, 10 iterations"}


def reference_arm(args, rank):
    if rank != 0:
        return 0
    exe = reference_timer_path()
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/hpcg_ref_timer was not built "
                          "(the reference tree was absent at build time)"}))
        return 0
    steps, warm = max(1, args.steps), max(0, args.warmup)
    iters = reference_iters_for(args.ref_n, 120.0, steps + warm)
    r = run_reference_sample(args.ref_n, iters, steps, warm)
    val = r["flops_per_call"] / r["mean_s"] / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 4), "unit": "GFLOP/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": warm, "ms_per_step": round(r["mean_s"] * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"HPCG CG_ref, {args.ref_n}^3 sample (the reference cannot generate 512^3: "
                               f"3.6e9 nonzeros overflow its int local_int_t), {iters} iterations per step",
                   "grid": [args.ref_n] * 3, "mg_levels": 4, "iters_per_step": iters},
        "cpu_baseline": {"value": round(val, 4), "unit": "GFLOP/s", "cores": r["threads"], "kind": "reference",
                         "sample": f"{args.ref_n}^3, {iters} CG_ref iterations per step"},
        "e2e": {"value": round(val, 4), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def committed_traffic():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    path = os.path.join(HERE, "profiles", "gs_phase_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------

RHS_SEED = 0x48504347


def uniform_rhs(nrow, device):
    """b ~ U[-1, 1], FP64, from a fixed seed (numpy PCG64), built on the host."""
    import numpy as np
    import torch
    b = np.random.Generator(np.random.PCG64(RHS_SEED)).uniform(-1.0, 1.0, nrow)
    return torch.from_numpy(b).to(device)


def timed(lib_stream, fn):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(lib_stream)
    out = fn()
    e1.record(lib_stream)
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1) * 1e-3


def adjoint_timing(dev, n=128, tol=1e-10):
    """Perturbed symmetric stencil at n^3: forward solve to `tol` (after the
    first-use tuning), loss 0.5 ||x - x_target||^2, then the implicit adjoint
    (dL/db and dL/da)."""
    import torch
    from hpcg_b200 import binding as B
    from hpcg_b200 import perturbed as PT
    nrow = n ** 3
    P = B.Problem.generate(n, n, n, 4, dev)
    try:
        vals = torch.from_numpy(PT.perturbed_values(n, n, n)).to(f"cuda:{dev}")
        P.set_values(0, vals)
        b = torch.from_numpy(PT.rhs_uniform(nrow)).to(f"cuda:{dev}")
        xt = torch.from_numpy(PT.target_normal(nrow)).to(f"cuda:{dev}")
        lib_stream = torch.cuda.ExternalStream(B.stream(dev), device=dev)
        x = torch.zeros_like(b)
        P.CG(b, x, 1, tol, True)  # untimed: tuning and the CG graph, which the adjoint then reuses
        x.zero_()
        (it_f, nr, nr0), t_f = timed(lib_stream, lambda: P.CG(b, x, 2000, tol, True))
        g = x - xt
        gb = torch.empty_like(b)
        gv = torch.empty_like(vals)
        it_a, t_a = timed(lib_stream, lambda: P.adjoint(x, g, 2000, tol, gb, gv))
        return {"grid": [n, n, n], "tolerance": tol, "forward": {"iters": it_f, "seconds": round(t_f, 4)},
                "adjoint": {"iters": it_a, "seconds": round(t_a, 4)},
                "loss": float(0.5 * torch.sum((x - xt) ** 2)), "grad_b_norm": float(torch.linalg.vector_norm(gb)),
                "grad_values_norm": float(torch.linalg.vector_norm(gv))}
    finally:
        P.free()


def multi_rhs(dev, n=256, k=8, tol=1e-9, max_iter=2000):
    """k systems b_j ~ U[-1, 1] (seeded) on the n^3 problem: the lockstep solver
    (hpcg_b200_cg_multi) against k one-at-a-time solves (hpcg_b200_cg)."""
    import numpy as np
    import torch
    from hpcg_b200 import binding as B
    nrow = n ** 3
    P = B.Problem.generate(n, n, n, 4, dev)
    try:
        lib_stream = torch.cuda.ExternalStream(B.stream(dev), device=dev)
        rng = np.random.Generator(np.random.PCG64(RHS_SEED))
        b = torch.from_numpy(rng.uniform(-1.0, 1.0, (k, nrow))).to(f"cuda:{dev}")
        x = torch.zeros_like(b)
        P.CG_multi(b[:, :], x, 1, tol)  # first use allocates the multi-system vectors
        x.zero_()
        (ni, nr, nr0), t_multi = timed(lib_stream, lambda: P.CG_multi(b, x, max_iter, tol))
        xs = torch.zeros(nrow, dtype=torch.float64, device=f"cuda:{dev}")
        P.CG(b[0].contiguous(), xs, 1, tol, True)  # untimed: the single-system tuning and CG graph
        iters_single, t_single = [], 0.0
        for j in range(k):
            xs.zero_()
            bj = b[j].contiguous()
            (it, _, _), t = timed(lib_stream, lambda: P.CG(bj, xs, max_iter, tol, True))
            iters_single.append(it)
            t_single += t
        return {"grid": [n, n, n], "rhs": k, "tolerance": tol,
                "lockstep": {"iters": [int(v) for v in ni], "seconds": round(t_multi, 3),
                             "solves_per_s": round(k / t_multi, 3),
                             "max_scaled_residual": float(np.max(nr / nr0))},
                "one_at_a_time": {"iters": iters_single, "seconds": round(t_single, 3),
                                  "solves_per_s": round(k / t_single, 3)},
                "speedup": round(t_single / t_multi, 3)}
    finally:
        P.free()


def batched(dev, count=16, tol=1e-9, max_iter=2000):
    """`count` problems with grid sides drawn by seed from {32, 48, 64, 96, 128}:
    one batched solve (hpcg_b200_batch_cg_mixed) against one-at-a-time solves
    (hpcg_b200_cg_mixed), FP64 flexible CG around the FP32 V-cycle, each
    problem's own right-hand side, to `tol`."""
    import numpy as np
    import torch
    from hpcg_b200 import binding as B
    rng = np.random.Generator(np.random.PCG64(RHS_SEED))
    sides = [32, 48, 64, 96, 128]
    dims = [tuple(int(v) for v in rng.choice(sides, 3)) for _ in range(count)]
    bt = B.Batch(dims, dev)
    try:
        lib_stream = torch.cuda.ExternalStream(B.stream(dev), device=dev)
        bs = [torch.from_numpy(p.get_rhs()).to(f"cuda:{dev}") for p in bt.problems]
        xs = [torch.zeros_like(b) for b in bs]
        bt.CG_mixed(bs, xs, 1, tol)  # builds the graph
        for x in xs:
            x.zero_()
        (ni, nr, nr0), t_batch = timed(lib_stream, lambda: bt.CG_mixed(bs, xs, max_iter, tol))
        iters_single, t_single = [], 0.0
        for p, b in zip(bt.problems, bs):
            x = torch.zeros_like(b)
            p.CG_mixed(b, x, 1, tol)  # first use prepares the FP32 copies
            x.zero_()
            (it, _, _), t = timed(lib_stream, lambda: p.CG_mixed(b, x, max_iter, tol))
            iters_single.append(it)
            t_single += t
        form = {0: "one launch per step, register phases", 1: "one launch per step, bulk-copy phases",
                2: "one cooperative launch per iteration"}[bt.form()]
        return {"problems": count, "dims": dims, "tolerance": tol, "form": "FP64 flexible CG, FP32 V-cycle",
                "iteration_form": form,
                "batched": {"iters": [int(v) for v in ni], "seconds": round(t_batch, 4),
                            "solves_per_s": round(count / t_batch, 2),
                            "max_scaled_residual": float(np.max(nr / nr0))},
                "one_at_a_time": {"iters": iters_single, "seconds": round(t_single, 4),
                                  "solves_per_s": round(count / t_single, 2)},
                "speedup": round(t_single / t_batch, 3)}
    finally:
        bt.free()


def mixed_vs_fp64(P, b, lib_stream, tol, max_iter=2000, profile_iters=20):
    """Time to a relative residual `tol` from x = 0: FP64 PCG (hpcg_b200_cg) against
    FP64 flexible PCG around the FP32 V-cycle (hpcg_b200_cg_mixed), both with
    their set-up (tuning, the FP32 copies) done beforehand. Then
    `profile_iters` more FP32 iterations with the launch profiler on give the
    level-0 FP32 Gauss-Seidel phases' achieved bandwidth."""
    import torch
    from hpcg_b200 import binding as B
    from hpcg_b200 import metrics
    n = b.numel()
    x64 = torch.zeros_like(b)
    (it64, nr64, nr064), t64 = timed(lib_stream, lambda: P.CG(b, x64, max_iter, tol, True))
    x32 = torch.zeros_like(b)
    P.CG_mixed(b, x32, 1, tol)  # untimed: builds and tunes the FP32 copies, as the FP64 path was before
    x32.zero_()
    (it32, nr32, nr032), t32 = timed(lib_stream, lambda: P.CG_mixed(b, x32, max_iter, tol))
    err = float(torch.linalg.vector_norm(x32 - x64) / torch.linalg.vector_norm(x64))
    ax = torch.zeros_like(b)
    P.ComputeSPMV(x32, ax)
    torch.cuda.synchronize()
    res = B.ComputeDotProduct(n, b - ax, b - ax) ** 0.5 / B.ComputeDotProduct(n, b, b) ** 0.5
    dev = b.device.index or 0
    B.profile(True, dev)
    x32.zero_()
    torch.cuda.synchronize()
    P.CG_mixed(b, x32, profile_iters, 0.0)
    fu_ms, fu_l, fu_rows = B.profile_read(B.PROF_GS32_FULL, dev)
    fi_ms, fi_l, fi_rows = B.profile_read(B.PROF_GS32_FIRST, dev)
    B.profile(False, dev)
    peak, _ = measured_peak_hbm()
    pack = P.level_pack_width(0) if P.level_config(0)["gs32"] == 10 else 0
    full_gbs = metrics.gs_phase_bytes(fu_rows, n, vb=4, pack=pack) / (fu_ms * 1e-3) / 1e9 if fu_ms else None
    first_gbs = metrics.first_sweep_bytes(fi_rows, vb=4) / (fi_ms * 1e-3) / 1e9 if fi_ms else None
    return {"fp64": {"iters": it64, "seconds": round(t64, 3), "scaled_residual": nr64 / nr064},
            "fp32_vcycle": {"iters": it32, "seconds": round(t32, 3), "scaled_residual": nr32 / nr032,
                            "true_residual": res},
            "time_ratio": round(t32 / t64, 4), "x_rel_diff_vs_fp64": err,
            "fp32_level0_phases": {
                "iters_profiled": profile_iters,
                "full_ms_per_iter": round(fu_ms / profile_iters, 3),
                "full_gbs": round(full_gbs, 1) if full_gbs else None,
                "full_frac": round(full_gbs / peak, 4) if full_gbs else None,
                "first_ms_per_iter": round(fi_ms / profile_iters, 3),
                "first_gbs": round(first_gbs, 1) if first_gbs else None,
                "bytes_per_row": {"full": round(metrics.gs_phase_bytes(1, 8, vb=4, pack=pack), 3),
                                  "first_sweep": 130},
                "column_form": pack}}


def gpu_launches_per_set(iters, nlevels=4, rtz_pass=False, wave=(0, 0, 0, 0)):
    """Kernels the library launches for one CG call (its own kernels only).
    rtz_pass: r'z runs as its own dot kernel (level 0 on the packed bulk-copy
    phases) instead of coming out of the post-smoother. wave[l]: level l runs
    its sweeps from nonzero x as one wavefront launch each (the pre-smoother's
    8 first-sweep phases, then 1 + 1 + 1 launches instead of 7 + 8 + 7)."""
    def sweeps(l):
        return 8 + 3 if l < len(wave) and wave[l] else 15 * 2
    # per non-coarsest level: pre and post symmetric sweeps, residual-restriction, prolongation
    coarsest = 8 + 1 if nlevels - 1 < len(wave) and wave[nlevels - 1] else 15  # one symmetric sweep from zero
    per_mg = sum(sweeps(l) + 2 for l in range(nlevels - 1)) + coarsest
    # r'z finalize (its partials come out of the post-smoother, or out of a dot
    # kernel), p update with the previous iteration's x update (k > 1), SpMV +
    # finalize, r update + finalize
    per_iter = per_mg + 1 + 1 + 2 + 2 + (1 if rtz_pass else 0)
    first_iter_adjust = -1  # k = 1 copies z to p instead of the update kernel
    loads_stores = 2 + 1    # b and x gathered in, x scattered out
    preamble = 3            # SpMV, r = b - Ax with r'r, finalize
    last_x = 1              # the last iteration's x update, after the loop
    return iters * per_iter + first_iter_adjust + loads_stores + preamble + last_x


def b200_arm(args, rank, world, local_rank):
    import torch
    from hpcg_b200 import binding as B
    from hpcg_b200 import metrics

    dev = local_rank
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", dev))

    n = args.n
    nrow = n ** 3
    t_setup = time.perf_counter()
    P = B.Problem.generate(n, n, n, 4, dev)
    t_setup = time.perf_counter() - t_setup
    b = torch.empty(nrow, dtype=torch.float64, device=f"cuda:{dev}")
    x = torch.zeros(nrow, dtype=torch.float64, device=f"cuda:{dev}")
    P.get_rhs(b)
    torch.cuda.synchronize()
    lib_stream = torch.cuda.ExternalStream(B.stream(dev), device=dev)

    def step(bv, xv):
        if xv.is_cuda:
            xv.zero_()
            torch.cuda.current_stream().synchronize()
        else:
            xv.zero_()
        return P.CG(bv, xv, args.iters, 0.0, True)

    # warm-up: tuning, graph construction, clocks settling
    for _ in range(args.warmup):
        step(b, x)
    B.profile(True, dev)
    step(b, x)  # the kernel-by-kernel loop once, untimed
    B.profile(False, dev)

    # the timed sets, kernel by kernel with the library's launch profiler on: CUDA
    # events on the library stream around the timed kernel classes (roofline)
    B.profile(True, dev)
    clocks = ClockSampler(dev)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(lib_stream)
    res = None
    for _ in range(args.steps):
        res = step(b, x)
    e1.record(lib_stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    gs_ms, gs_launch, gs_rows = B.profile_read(B.PROF_GS_FULL, dev)
    sp_ms, sp_launch, sp_rows = B.profile_read(B.PROF_SPMV, dev)
    gf_ms, gf_launch, gf_rows = B.profile_read(B.PROF_GS_FIRST, dev)
    rs_ms, rs_launch, rs_rows = B.profile_read(B.PROF_RESTRICT, dev)
    ws_ms, ws_launch, ws_rows = B.profile_read(B.PROF_GS_SWEEP, dev)
    B.profile(False, dev)
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # the same sets with the profiler off: the library's default path, the CG
    # loop as one CUDA graph (conditional while node), as e2e runs it
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    g0 = torch.cuda.Event(enable_timing=True)
    g1 = torch.cuda.Event(enable_timing=True)
    g0.record(lib_stream)
    for _ in range(args.steps):
        step(b, x)
    g1.record(lib_stream)
    torch.cuda.synchronize()
    ms_graph = g0.elapsed_time(g1)
    if dist:
        t = torch.tensor([ms_graph], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_graph = float(t.item())

    flops_step = metrics.hpcg_flops(n, n, n, args.iters)
    value = flops_step * args.steps * world / (ms * 1e-3) / 1e9
    # the iteration's algorithmic bytes as the library's kernels move them,
    # with each level's column index as stored (8-bit or 16-bit offsets, or
    # 32-bit columns)
    packs = tuple(P.level_pack_width(l) for l in range(4))
    # r'z rides on the post-smoother except on 8-bit / 16-bit offset records
    rtz_fused = not (P.level_config(0)["gs"] == 10 and packs[0] in (1, 2))
    waves = tuple(P.level_wavefront(l) for l in range(4))
    bytes_iter = metrics.iteration_bytes(n, n, n, vb=8, pack=packs, rtz_fused=rtz_fused, wave=waves)
    hbm_gbs = bytes_iter * args.iters * args.steps / (ms * 1e-3) / 1e9  # per GPU

    # end to end through the C ABI with pinned host vectors
    e2e = None
    if not args.no_e2e:
        bh = b.cpu().pin_memory()
        xh = torch.zeros(nrow, dtype=torch.float64).pin_memory()

        def e2e_ms():
            step(bh, xh)
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            f0 = torch.cuda.Event(enable_timing=True)
            f1 = torch.cuda.Event(enable_timing=True)
            f0.record(lib_stream)
            for _ in range(args.steps):
                step(bh, xh)
            f1.record(lib_stream)
            torch.cuda.synchronize()
            t_ms = f0.elapsed_time(f1)
            if dist:
                t = torch.tensor([t_ms], dtype=torch.float64, device=f"cuda:{dev}")
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                t_ms = float(t.item())
            return t_ms

        # every step moves b and x in and x out: the library's reuse of an
        # unchanged b and a zero x is switched off for this leg
        P.set_host_reuse(False)
        ems = e2e_ms()
        P.set_host_reuse(True)
        rms = e2e_ms()
        e2e = {"value": round(flops_step * args.steps * world / (ems * 1e-3) / 1e9, 3), "unit": "GFLOP/s",
               "h2d_bytes_per_step": 2 * nrow * 8, "d2h_bytes_per_step": nrow * 8 + 64,
               "ms_per_step": round(ems / args.steps, 3),
               "with_host_reuse": {"value": round(flops_step * args.steps * world / (rms * 1e-3) / 1e9, 3),
                                   "ms_per_step": round(rms / args.steps, 3), "h2d_bytes_per_step": 0,
                                   "d2h_bytes_per_step": nrow * 8 + 64,
                                   "note": "the same b every step and a zero x, as the reference's timed loop "
                                           "passes them: b compared on the host, x zeroed on the device"}}

    mixed = None
    if not args.no_mixed:
        mixed = {"tolerance": args.mixed_tol}
        if args.mixed_rhs in ("hpcg", "both"):
            mixed["rhs_hpcg"] = mixed_vs_fp64(P, b, lib_stream, args.mixed_tol)
        if args.mixed_rhs in ("uniform", "both"):
            mixed["rhs_uniform"] = mixed_vs_fp64(P, uniform_rhs(nrow, f"cuda:{dev}"), lib_stream, args.mixed_tol)
        # the floor of the time ratio: the two forms' algorithmic bytes per
        # iteration (both bandwidth-bound at about the same efficiency)
        packs = tuple(P.level_pack_width(l) for l in range(4))
        b64 = metrics.iteration_bytes(n, n, n, vb=8, pack=packs, rtz_fused=rtz_fused, wave=waves)
        b32 = metrics.iteration_bytes(n, n, n, vb=4, pack=packs)
        mixed["byte_floor_ratio"] = round(b32 / b64, 4)
        mixed["bytes_per_iter"] = {"fp64": b64, "fp32_vcycle": b32, "column_form": list(packs)}

    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_timing(dev)
    multi = None
    if not args.no_multi:
        multi = multi_rhs(dev, n=args.multi_n)
    batch = None
    if not args.no_batch:
        batch = batched(dev)
    # the copy side's ceiling on level 0's tiles: the FP64 phases' pipeline over
    # the whole matrix with consumers that hand each stage straight back (the
    # fastest of three launches; outside every timed region)
    probe = None
    try:
        pms, pbytes = min(P.stream_probe(0) for _ in range(3))
        probe = {"gbs": round(pbytes / (pms * 1e-3) / 1e9, 1), "ms": round(pms, 4), "bytes": pbytes,
                 "note": "hpcg_b200_stream_probe: level 0's values and column index, every 128-row tile "
                         "through the Gauss-Seidel phases' copy pipeline, no consumer work"}
    except B.HpcgError as ex:
        probe = {"gbs": None, "error": str(ex)[:200]}

    line = None
    tuning = [P.level_config(l) for l in range(4)]
    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        gs_cfg = tuning[0]["gs"]
        pack0 = P.level_pack_width(0)
        gs_pack = pack0 if gs_cfg == 10 else 0
        mv_pack = pack0 if tuning[0]["spmv"] == 7 else 0
        gs_packed = gs_pack > 0
        gs_bytes = metrics.gs_phase_bytes(gs_rows, nrow, pack=gs_pack)
        achieved = gs_bytes / (gs_ms * 1e-3) / 1e9 if gs_ms > 0 else None
        kernel = (f"k_gs_bulk<double,double,false> (level 0, configuration {gs_cfg}"
                  f"{', packed columns, ' + COLUMN_FORMS[gs_pack] if gs_pack else ''})" if gs_cfg == 10 else
                  f"k_gs_phase<double,double,false> (level 0, configuration {gs_cfg})")
        tr = committed_traffic()
        traffic = None
        if (tr and tr.get("n") == n and tr.get("config") == gs_cfg and int(tr.get("pack", 0)) == gs_pack
                and gs_launch and tr.get("form", "phase") == "phase"):
            traffic = tr.get("bytes_per_launch")
        # level 0's sweeps as wavefront launches: then the dominant kernel
        ws_bytes = metrics.wave_sweep_bytes(ws_rows, nrow, pack=pack0) if ws_launch else 0.0
        wave_line = None
        if ws_launch:
            wave_line = {"launches": ws_launch, "avg_ms": round(ws_ms / ws_launch, 4),
                         "gbs": round(ws_bytes / (ws_ms * 1e-3) / 1e9, 1) if ws_ms else None,
                         "bytes_per_row": metrics.wave_sweep_bytes(nrow, nrow, pack=pack0) / nrow,
                         "levels": list(waves)}
        phase_ms = gs_ms  # the level-0 phases launched one by one (kernel_ms_per_iter)
        if ws_launch and ws_ms > gs_ms:
            gs_bytes, gs_ms, gs_launch = ws_bytes, ws_ms, ws_launch
            achieved = ws_bytes / (ws_ms * 1e-3) / 1e9 if ws_ms > 0 else None
            kernel = (f"k_gs_wave<double,{pack0}> (a whole level-0 sweep per launch, wavefront over z pairs, "
                      f"column form {pack0})")
            traffic = None
            if (tr and tr.get("n") == n and tr.get("form") == "wave" and int(tr.get("pack", 0)) == pack0):
                traffic = tr.get("bytes_per_launch")
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"HPCG CG set: {args.iters} preconditioned CG iterations, {n}^3 grid, "
                                   f"4 MG levels, 27-point stencil, 8-colour SYMGS, FP64",
                       "grid": [n, n, n], "rows": nrow, "mg_levels": 4, "iters_per_step": args.iters,
                       "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (43 GB matrix)",
                       "setup_s": round(t_setup, 3)},
            "graph_loop": {"value": round(flops_step * args.steps * world / (ms_graph * 1e-3) / 1e9, 3),
                           "ms_per_step": round(ms_graph / args.steps, 3),
                           "note": "same sets, profiler off: the CG loop as one CUDA graph, the library's "
                                   "default path (e2e runs it)"},
            "iteration": {"bytes": bytes_iter, "gbs": round(hbm_gbs, 1), "frac": round(hbm_gbs / peak, 4),
                          "model": "metrics.iteration_bytes: every kernel of a CG iteration streaming its data "
                                   "once, each level's column index as stored",
                          "column_form": list(packs),
                          "compulsory_4byte_index_bytes": metrics.compulsory_bytes(n, n, n)},
            "packed_index_bytes": [P.level_packed(l) for l in range(4)],
            "final_scaled_residual": res[1] / res[2] if res and res[2] else None,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None, "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4) if achieved else None,
                         "traffic": traffic, "kernel": kernel,
                         "peak_kind": f"{peak_kind} (MEASURED_PEAKS hbm_gbs)" if peak_kind == "measured"
                         else peak_kind, "launches": gs_launch, "avg_launch_ms": round(gs_ms / max(gs_launch, 1), 4),
                         "bytes_per_launch": gs_bytes / max(gs_launch, 1)},
            "spmv": {"launches": sp_launch, "avg_ms": round(sp_ms / max(sp_launch, 1), 4),
                     "gbs": round(metrics.spmv_bytes(sp_rows, pack=mv_pack) / (sp_ms * 1e-3) / 1e9, 1)
                     if sp_ms else None, "column_form": mv_pack},
            "first_sweep_gbs": round(metrics.first_sweep_bytes(gf_rows) / (gf_ms * 1e-3) / 1e9, 1) if gf_ms else None,
            "kernel_ms_per_iter": {
                "gs_full_l0": round(phase_ms / (args.iters * args.steps), 3),
                "gs_first_l0": round(gf_ms / (args.iters * args.steps), 3),
                "spmv_l0": round(sp_ms / (args.iters * args.steps), 3),
                "restrict_l0": round(rs_ms / (args.iters * args.steps), 3),
                "gs_sweeps_l0": round(ws_ms / (args.iters * args.steps), 3) if wave_line else 0.0,
                "iteration": round(ms / (args.iters * args.steps), 3)},
            "gpu_launches": gpu_launches_per_set(args.iters, rtz_pass=gs_packed and gs_pack != 3,
                                                 wave=waves) * args.steps,
            "clocks": clk,
        }
        if wave_line:
            line["wavefront_sweeps"] = wave_line
        if probe:
            line["stream_probe"] = probe
        if e2e:
            line["e2e"] = e2e
        if mixed:
            line["mixed_precision"] = mixed
        if adjoint:
            line["adjoint"] = adjoint
        if multi:
            line["multi_rhs"] = multi
        if batch:
            line["batched"] = batch
        if not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline(args)
            except Exception as ex:  # reported, not fatal
                line["cpu_baseline"] = {"value": None, "error": str(ex)[:200]}
    if line:
        line["config"]["autotuned"] = tuning
        line["config"]["level_config"] = P.level_config_string()
    P.free()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if line:
        print(json.dumps(line))
    return 0


def shard_launches_per_set(iters, nlevels=4, halo=True, rtz_fused=True):
    """Kernels one rank launches for one sharded CG call (its own kernels only).
    halo: the rank has neighbours (a halo pack before each exchange);
    rtz_fused: r'z comes from the post-smoother (its store and the rank fold)
    instead of a dot kernel of its own (dot, store, fold)."""
    pack = 1 if halo else 0
    # per non-coarsest level: first sweep (15 phases), halo pack, restriction,
    # prolongation, halo pack, post sweep (15 phases); coarsest: 15 phases
    per_mg = (15 + pack + 1 + 1 + pack + 15) * (nlevels - 1) + 15
    # r'z, p update with the previous x update, halo pack, SpMV + store + fold, r update + store + fold
    per_iter = per_mg + (2 if rtz_fused else 3) + 1 + pack + 3 + 3
    # k = 1 copies p instead; the last x update; loads/stores; preamble pack + SpMV, residual, store, fold
    return iters * per_iter - 1 + 1 + 3 + (pack + 4)


def shard_arm(args, rank, world, local_rank):
    """One rank of the decomposition over `world` GPUs (NCCL halo + allreduce)."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from hpcg_b200 import binding as B
    from hpcg_b200 import metrics

    dev = local_rank
    torch.cuda.set_device(dev)
    if world == 1:  # --decomposed on one GPU, without a launcher
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29533")
        os.environ.setdefault("RANK", "0")
        os.environ.setdefault("WORLD_SIZE", "1")
    dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", dev))
    n = args.n
    nrow = n ** 3
    npx, npy, npz = B.process_grid(world)
    t_setup = time.perf_counter()
    P = B.Problem.generate_rank(n, n, n, npx, npy, npz, rank, 4, dev)
    obj = [B.comm_unique_id() if rank == 0 else None]
    dist.broadcast_object_list(obj, src=0)
    C = B.Comm.nccl(obj[0], world, rank, P)
    t_setup = time.perf_counter() - t_setup
    b = torch.from_numpy(P.get_rhs()).to(f"cuda:{dev}")
    x = torch.zeros(nrow, dtype=torch.float64, device=f"cuda:{dev}")
    lib_stream = torch.cuda.ExternalStream(B.stream(dev), device=dev)

    def step(bv, xv):
        xv.zero_()
        if xv.is_cuda:
            torch.cuda.current_stream().synchronize()
        return C.CG([bv], [xv], args.iters, 0.0, True)

    def timed_steps(bv, xv):
        dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lib_stream)
        r = None
        for _ in range(args.steps):
            r = step(bv, xv)
        e1.record(lib_stream)
        torch.cuda.synchronize()
        dist.barrier()
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()), r

    for _ in range(args.warmup):
        step(b, x)
    B.profile(True, dev)
    clocks = ClockSampler(dev)
    clocks.start()
    ms, res = timed_steps(b, x)
    clk = clocks.stop()
    gs_ms, gs_launch, gs_rows = B.profile_read(B.PROF_GS_FULL, dev)
    B.profile(False, dev)
    gflop = metrics.hpcg_flops(npx * n, npy * n, npz * n, args.iters) * args.steps / 1e9
    value = gflop / (ms * 1e-3)
    e2e = None
    if not args.no_e2e:
        bh = b.cpu().pin_memory()
        xh = torch.zeros(nrow, dtype=torch.float64).pin_memory()
        step(bh, xh)
        ems, _ = timed_steps(bh, xh)
        e2e = {"value": round(gflop / (ems * 1e-3), 3), "unit": "GFLOP/s",
               "h2d_bytes_per_step": world * 2 * nrow * 8, "d2h_bytes_per_step": world * nrow * 8,
               "ms_per_step": round(ems / args.steps, 3)}
    line = None
    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        gs_cfg = P.level_config(0)["gs"]
        gs_pack = P.level_pack_width(0) if gs_cfg == 10 else 0
        gs_bytes = metrics.gs_phase_bytes(gs_rows, nrow, pack=gs_pack)
        achieved = gs_bytes / (gs_ms * 1e-3) / 1e9 if gs_ms > 0 else None
        kernel = (f"k_gs_bulk<double,double,false> (level 0 of rank 0, configuration 10"
                  f"{f', column form {gs_pack}' if gs_pack else ''})" if gs_cfg == 10 else
                  f"k_gs_phase<double,double,false> (level 0 of rank 0, configuration {gs_cfg})")
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"HPCG CG set over {world} ranks: {args.iters} preconditioned CG iterations, "
                                   f"{n}^3 block per rank, 4 MG levels, 27-point stencil, 8-colour SYMGS, FP64",
                       "grid": [npx * n, npy * n, npz * n], "local_grid": [n, n, n], "rows": world * nrow,
                       "process_grid": [npx, npy, npz], "mg_levels": 4, "iters_per_step": args.iters,
                       "parallelism": f"halo{world}: NCCL halo exchange + allreduce",
                       "l2": "inputs larger than L2 (43 GB matrix per rank)", "setup_s": round(t_setup, 3)},
            "final_scaled_residual": res[1] / res[2] if res and res[2] else None,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None, "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4) if achieved else None, "traffic": None,
                         "kernel": kernel,
                         "peak_kind": peak_kind, "launches": gs_launch},
            "gpu_launches": shard_launches_per_set(args.iters, halo=world > 1,
                                                   rtz_fused=not (gs_cfg == 10 and gs_pack in (1, 2))) * args.steps,
            "clocks": clk,
        }
        if e2e:
            line["e2e"] = e2e
    C.free()
    P.free()
    dist.barrier()
    dist.destroy_process_group()
    if line:
        print(json.dumps(line))
    return 0


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.case:
        return profile_case(args.case)
    if args.vcycle:
        return profile_vcycle(args.vcycle)
    if args.impl == "reference":
        return reference_arm(args, rank)
    if (world > 1 and not args.replicas) or args.decomposed:
        return shard_arm(args, rank, world, local_rank)
    return b200_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
