"""Benchmark of the MAPP force-field hot path on B200.

Metric: DMD site-force evaluations per second (owned sites x force_calc calls
/ device seconds) for the binary DMD_I system of FCC 20^3 = 32000 sites
(a = 3.58 A, alpha = 1/w^2 with w ~ U(0.08, 0.15) A, c_A ~ Beta(2,2),
n = 3 Gauss-Hermite nodes, T = 600 K), synthetic seeded inputs.

One step = one ForceField::force_calc(1, en_st) of the whole system (both
passes, embedding and the energy/virial reduction), inputs resident in HBM;
L2 is flushed (256 MiB write) before every timed step.  `e2e` repeats the step
through the C ABI with host buffers: owned x and c copied in (update_0 +
update(c)), forces and en_st copied out.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank relaxes its own independent system (replicas, no
collective on the data path); `value` sums the sites of all ranks over the
slowest rank's device time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DMD site-force evals/s, surrogate & FP32 vs FP64 on 1 B200 at max|dF|<=1e-4 eV/A"
UNIT = "site-force evals/s"
WORKLOAD = dict(n=20, a=3.58, sigma=0.0, style="DMD_I")
# flops of one evaluation of the learned form's network 4 -> 64 -> 64 -> 64 -> 6
MLP_FLOPS_PER_ROW = 2 * (4 * 64 + 64 * 64 + 64 * 64 + 64 * 6)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cells", type=int, default=WORKLOAD["n"], help="FCC cells per edge (default 20 -> 32000 sites)")
    p.add_argument("--cpu-reps", type=int, default=0, help="reference force_calc calls per CPU process (0: auto)")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU reference timing")
    p.add_argument("--skip-forms", action="store_true", help="skip the FP32, learned and batched forms (profiling runs)")
    p.add_argument("--form", default="fp64", choices=["fp64", "fp32", "mlp"],
                   help="form of the timed force_calc steps (fp32 / mlp imply --skip-forms; for profiling)")
    p.add_argument("--eam-cells", type=int, default=0,
                   help="instead: time EAM force_calc (the MD crystal's potential) on FCC n^3 atoms (profiling)")
    p.add_argument("--clock", default="", choices=["", "adams", "bdf"],
                   help="instead: run only the Adams (32000 sites) or BDF (--cells, default 32000 sites) clock line, "
                        "without the CPU reference (profiling)")
    return p.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workload_config(args, extra=None):
    c = {"workload": f"DMD_I binary FCC {args.cells}^3 = {4 * args.cells ** 3} sites, a=3.58 A, "
                     "w~U(0.08,0.15) A (alpha=1/w^2), c_A~Beta(2,2), n_quad=3, T=600 K, "
                     "r_crd=3.0, alpha_min=20, alpha_max=1000, skin 0.5 A",
         "sites": 4 * args.cells ** 3, "species": 2, "step": "force_calc(st_clc=1)",
         "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas" if args.gpus > 1 else "1 gpu"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
# CPU reference (the reference's own force_calc through oracle/_ref)
# ---------------------------------------------------------------------------
def cpu_reference(w, natms, reps, procs):
    from oracle import reference

    if not reference.available():
        return None
    cmds = []
    for p in range(procs):
        d = tempfile.mkdtemp(prefix=f"mapp_cpu{p}_")
        # one untimed call first: the reference allocates its per-pair buffers on the first force_calc
        rr = reference.RefRun(w, workdir=d).time("force", 1, tag="warm").time("force", reps, tag="t")
        # reuse RefRun's command-file writer without running it
        cmds.append(rr)
    t0 = time.time()
    threads, results = [], [None] * procs

    def run(k):
        results[k] = cmds[k].run(timeout=1800)

    for k in range(procs):
        th = threading.Thread(target=run, args=(k,))
        th.start()
        threads.append(th)
    for th in threads:
        th.join()
    wall = time.time() - t0
    per = [r["t"]["meta"]["time_force"][1] for r in results]
    value = sum(natms * reps / t for t in per)
    return dict(value=value, per_proc_s=per, wall=wall)


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from mapp_b200 import fixtures as fx

    d = tempfile.mkdtemp(prefix="mapp_bench_ref_")
    w = fx.write_workload(d, "dmd", n=args.cells, a=WORKLOAD["a"], sigma=WORKLOAD["sigma"], style="DMD_I")
    natms = w["cfg"].natms
    procs = os.cpu_count() or 1
    reps = max(1, args.cpu_reps or 2)
    values = []
    # warm-up calls are part of each process's init (first force_calc); time K steps of `reps` calls
    steps = max(1, min(args.steps, 3))
    for _ in range(steps):
        r = cpu_reference(w, natms, reps, procs)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference harness oracle/_ref/mapp_ref_harness not built"}))
            return 0
        values.append(r["value"])
    value = float(np.median(values))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": natms / value * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
                         "sample": f"{procs} concurrent single-rank reference processes x {reps} force_calc calls "
                                   f"of the {natms}-site system each ({cpu_model()})"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# clocks sampling during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    """Samples SM clocks, power and throttle reasons with nvidia-smi while the
    timed work runs (reads only).  Each sample is one nvidia-smi query that
    exits by itself: a looping nvidia-smi writing to a file buffers its
    output, and a terminated one can leave the file empty."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device, period_s=0.1):
        self.device = device
        self.period = period_s
        self.rows = []
        self._stop = None
        self._thread = None

    def _run(self):
        cmd = ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits"]
        while not self._stop.is_set():
            try:
                out = subprocess.run(cmd, capture_output=True, text=True, timeout=5).stdout
            except (OSError, subprocess.SubprocessError):
                return
            for line in out.splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    self.rows.append(parts)
            self._stop.wait(self.period)

    def __enter__(self):
        import threading

        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._thread.join(timeout=10)

    def count(self):
        return len(self.rows)

    def summary(self):
        rows = list(self.rows)
        if not rows:
            return None

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None

        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in rows) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def job_max(value, device="cpu"):
    """Max over the ranks of a per-rank time; the value itself on one rank."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, steps, t_max_s, world):
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return world * units_per_rank * steps / t_max_s


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fp:
            return json.load(fp), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def measure_fp32_peak(n=8192, reps=5):
    """FP32 denominator for the precision form's compute view: cuBLAS SGEMM
    (torch.matmul in float32 with TF32 off, so the FP32 FMA pipe), n^3,
    best of reps, CUDA events."""
    import torch

    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(n, n, dtype=torch.float32, device="cuda")
    b = torch.randn(n, n, dtype=torch.float32, device="cuda")
    c = a @ b
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    torch.backends.cuda.matmul.allow_tf32 = old
    del a, b, c
    return 2.0 * n ** 3 / best / 1e12


def measure_fp64_peak(n=4096, reps=5):
    """FP64 denominator for the compute view of the roofline: cuBLAS DGEMM
    (torch.matmul in float64, n^3, 2 n^3 flops) on this GPU, best of reps,
    timed with CUDA events; MEASURED_PEAKS.json carries no FP64 figure."""
    import torch

    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = a @ b
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b, c
    return 2.0 * n ** 3 / best / 1e12


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def pass2_flops_per_pair(nt):
    """Algorithmic work of force pass 2 (the projection of the stored
    derivatives on the forces, ff_dmd_I.cpp:357-436) per half pair inside the
    smeared cut: about 25 flops per ordered species pair, nt^2 * 25 (100 for
    the binary system)."""
    return nt * nt * 25


def pass1_flops_per_pair(nt, nq):
    """Algorithmic FP64 work of force pass 1 per half pair inside the smeared
    cut, as counted for this workload's measurement: per ordered species pair
    about 10 flops of geometry and alpha combination plus about 22 per
    quadrature node (node offset, table index, two cubic evaluations, weighted
    sums), sqrt and division counted as one: nt^2 (10 + 22 nq), 304 for the
    binary n = 3 system."""
    return nt * nt * (10 + 22 * nq)


# Algorithmic bytes of force pass 1 per owned site: its share of the minimum
# traffic of one force evaluation (read x and alpha 40 B and c 16 B, write the
# densities E 16 B; the whole evaluation also writes f 40 B and dE 16 B, about
# 130 B per site).  Everything else pass 1 moves (the per-pair scratch, gathers
# of neighbour sites) is this implementation's traffic, seen in `traffic`.
PASS1_ALG_BYTES_PER_SITE = 72


def phase_times(s, f, steps, flush):
    """Mean per-kernel device times (pass 1, embedding, pass 2) of the DMD force
    call over `steps` calls (L2 flushed before each), in a loop of their own
    with the library's phase events on: those events cost the call a few
    microseconds each, so the throughput loops run without them."""
    import torch

    s.set_timing(2)
    t = [0.0, 0.0, 0.0, 0.0]
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        s.force_calc(1, f=f)
        for k, ph in enumerate(("force.pass1", "force.embed", "force.pass2", "force")):
            t[k] += s.last_time(ph)
    s.set_timing(1)
    return [v / steps for v in t]


def run_forms(args, s, mb, natms, f_dev, flush, t_dev):
    """Precision and learned forms on the same system: throughput, and errors
    against the plain FP64 form."""
    import torch

    f64_ref = f_dev.clone()
    s.force_calc(1, f=f64_ref)
    _, en64 = s.force_calc(1)
    s.set_form(mb.MG_FORM_FP32)
    f32 = torch.zeros_like(f_dev)
    for _ in range(args.warmup):
        s.force_calc(1, f=f32)
    t32 = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        _, en32 = s.force_calc(1, f=f32)
        t32 += s.last_time("force")
    t32_p1 = phase_times(s, f32, min(args.steps, 200), flush)[0]
    fp32_form = {"value": natms * args.steps / (t32 * 1e-3), "unit": UNIT, "ms_per_step": t32 / args.steps,
                 "pass1_ms": t32_p1, "pass1_note": "density pass, timed in a loop of its own with phase events on",
                 "max_abs_dF_eV_per_A": float((f32 - f64_ref).abs().max().item()),
                 "abs_dE_per_site_eV": abs(float(en32[0]) - float(en64[0])) / natms,
                 "speedup_vs_fp64": t_dev / t32,
                 "error_reference": "plain FP64 GPU form (itself within 1e-10 of the CPU oracle)"}
    s.set_form(mb.MG_FORM_FP64)

    # learned form: train on the GPU (2M quadrature-labelled samples, 20k Adam
    # steps of 4096, lr 1e-3 cosine), then force_calc with the network, the
    # quadrature fallback outside the training box and the 1% audit
    s.mlp_init(1.8, 5.0, 0.05, 0.20, seed=5)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mlp_loss = s.mlp_train(nsamples=2_000_000, steps=20_000, batch=4096, lr=1e-3, seed=11)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    s.set_form(mb.MG_FORM_MLP)
    fm = torch.zeros_like(f_dev)
    for _ in range(args.warmup):
        s.force_calc(1, f=fm)
    mlp_steps = max(10, min(args.steps, 400))
    tm = 0.0
    for _ in range(mlp_steps):
        flush.zero_()
        torch.cuda.synchronize()
        _, enm = s.force_calc(1, f=fm)
        tm += s.last_time("force")
    audit, audit_counts = s.mlp_audit()
    tm_p1 = phase_times(s, fm, min(mlp_steps, 100), flush)[0]
    mlp_form = {"value": natms * mlp_steps / (tm * 1e-3), "unit": UNIT, "ms_per_step": tm / mlp_steps,
                "steps": mlp_steps, "pass1_ms": tm_p1,
                "pass1_note": "network rows, fallback, network, audit and densities, timed in a loop of their own "
                              "with phase events on",
                "max_abs_dF_eV_per_A": float((fm - f64_ref).abs().max().item()),
                "abs_dE_per_site_eV": abs(float(enm[0]) - float(en64[0])) / natms,
                "speedup_vs_fp64": (t_dev / args.steps) / (tm / mlp_steps),
                "train_s": t_train, "train_final_loss": mlp_loss,
                "training": "2M samples, 20000 steps x 4096, Adam lr 1e-3 cosine, box r [1.8,5.0] w [0.05,0.20]",
                "audit_max_abs_err": {k: float(v) for k, v in zip(
                    ("phi", "rho", "dphi_dr", "drho_dr", "dphi_dalpha", "drho_dalpha"), audit)},
                "audited_rows": int(audit_counts[0]), "fallback_rows": int(audit_counts[1]),
                "error_reference": "plain FP64 GPU form (itself within 1e-10 of the CPU oracle)"}
    s.set_form(mb.MG_FORM_FP64)

    return {"fp32": fp32_form, "mlp": mlp_form}


def run_batched(mb, fx, device, ncells=512):
    """Batched form: 512 independent periodic DMD cells (site counts log-uniform
    in [500, 8000] as whole FCC cells, cubic or slab; per-cell mean c_A ~
    U(0.1, 0.9); w ~ U(0.08, 0.15) A) relaxed by L-BFGS (m = 5, stop at
    max|f| < 1e-5, the reference's energy tolerance 1e-8, or 60 halvings) in one
    graph launch, FP64 and FP32 force passes.  The second relaxation of each
    form is timed (its launch shapes come from the tuning cache)."""
    bdir = tempfile.mkdtemp(prefix="mapp_batch_")
    wb = fx.write_workload(bdir, "dmd", n=2, style="DMD_I")
    builder = mb.system_from_workload(wb, device=device)
    cells = fx.make_batch_cells(ncells, seed=2024)
    sites = int(sum(c.natms for c in cells))
    out = {"cells": ncells, "sites": sites, "m": 5, "fmax_tol": 1e-5, "energy_tol": 1e-8, "max_halvings": 60}
    for form, name in ((mb.MG_FORM_FP64, "fp64"), (mb.MG_FORM_FP32, "fp32")):
        B = mb.Batch(builder)
        for c in cells:
            B.add_cell(c)
        B.set_params(5, 10000, 1e-5, 1e-8, 60)
        B.set_form(form)
        B.set_tuning(True, os.path.join(bdir, "tune.txt"))
        first = B.relax()
        st = B.relax()
        res = [B.cell_result(k)[2] for k in range(ncells)]
        t = np.array([r["t_ms"] for r in res])
        mf = np.array([r["max_f"] for r in res])
        codes = np.bincount([r["code"] for r in res], minlength=6).tolist()
        out[name] = {
            # the lead figure: force evaluations of sites per second over the
            # whole relaxation; cells stop after about two iterations (their
            # forces are not the gradient of the energy the line search
            # tests), so relaxations/s does not measure relaxation work
            "site_evals_per_s": float(sum(r["evaluations"] * r["natms"] for r in res) / (st["relax_ms"] * 1e-3)),
            "relaxations_per_s": ncells / (st["relax_ms"] * 1e-3),
            "relaxations_per_s_with_build": ncells / ((st["relax_ms"] + st["build_ms"]) * 1e-3),
            "relax_ms": st["relax_ms"], "build_ms": st["build_ms"], "tune_ms_first_run": first["tune_ms"],
            "cell_time_ms_p50": float(np.percentile(t, 50)), "cell_time_ms_p99": float(np.percentile(t, 99)),
            "loop_iterations": st["iterations"], "cell_evaluations": st["evaluations"],
            "stop_codes": {"not_downhill": codes[1], "min_step": codes[3], "max_iter": codes[4],
                           "tolerance": codes[5]},
            "converged_max_f": st["converged"],
            "max_f_p50": float(np.median(mf)), "max_f_max": float(mf.max()),
            "iterations_p50": float(np.median([r["iterations"] for r in res])),
            "launch_shapes": {"bps1": st["bps1"], "bps2": st["bps2"], "lbfgs_threads": st["lbfgs_threads"],
                              "lbfgs_cluster": st["lbfgs_cluster"]},
            "rebuild_rounds": st["rebuild_rounds"]}
        B.close()
    out["note"] = ("cells stop on the reference's own criteria: its DMD forces are not the gradient of its "
                   "energy (quadrature identities; species-slot transposition in pass 2 for two species), so "
                   "no energy line search reaches max|f| < 1e-5")
    builder.close()
    return out


def run_e2e_client(mb, w, steps, device, warmup=3):
    """Runs mapp_b200/mapp_e2e (built with the library) on the workload w;
    returns its JSON line, or None when it is missing or fails."""
    client = os.path.join(os.path.dirname(os.path.abspath(mb.__file__)), "mapp_e2e")
    if not os.path.exists(client):
        return None
    cmd = [client, w["style"], w["cfg_path"], str(steps), str(warmup), str(device), str(w.get("skin", 0.5)),
           *w["coef"]]
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    except (OSError, subprocess.TimeoutExpired):
        return None
    if p.returncode != 0 or not p.stdout.strip():
        print(f"e2e client failed: {p.stderr.strip()[-300:]}", file=sys.stderr)
        return None
    return json.loads(p.stdout.strip().splitlines()[-1])


def run_batched_sharded(mb, fx, device, rank, world, ncells=512):
    """The batched form's 512 cells split over the job's GPUs
    (mapp_b200.shard): each rank relaxes its share (FP64, one graph launch,
    the second relaxation timed), the job time is the slowest rank's device
    time, the per-cell results are gathered on rank 0."""
    import torch

    from mapp_b200 import shard

    bdir = tempfile.mkdtemp(prefix=f"mapp_batch_sh{rank}_")
    wb = fx.write_workload(bdir, "dmd", n=2, style="DMD_I")
    builder = mb.system_from_workload(wb, device=device)
    cells = fx.make_batch_cells(ncells, seed=2024)
    st, local = shard.relax_sharded(builder, cells, rank, world, form=mb.MG_FORM_FP64,
                                    tuning_cache=os.path.join(bdir, "tune.txt"), warm=True)
    t_job_s = job_max(st["relax_ms"] * 1e-3, "cuda")
    evals = torch.tensor([float(sum(r["evaluations"] * r["natms"] for _, r in local))], dtype=torch.float64,
                         device="cuda")
    import torch.distributed as dist

    dist.all_reduce(evals)
    res = shard.gather_results(local, ncells)
    builder.close()
    if rank != 0:
        return None
    return {"cells": ncells, "ranks": world, "site_evals_per_s": float(evals.item()) / t_job_s,
            "relaxations_per_s": ncells / t_job_s, "job_relax_ms": t_job_s * 1e3,
            "rank0_cells": st["cells"], "rank0_sites": st["sites"],
            "cells_gathered": len(res), "assignment": "largest first to the least-loaded rank (by site count)"}


def run_large_forms(mb, fx, device, mlp_source):
    """The precision form on FCC 40^3 = 256000 sites (then the 256000-site
    workflow: 200 CG iterations in the precision form, 10 Adams steps, 100
    BDF steps of order at most 2) and the learned form on
    FCC 50^3 = 500000 sites (same distributions as the 32000-site system),
    each against the plain FP64 form on the same system: time per force call
    (L2 flushed before each), max|dF|, |dE|/site and, for the precision form,
    max|d mu| of the chemical potentials after c_d_calc.  The learned form
    reuses the network trained on the 32000-site system (same tables)."""
    import torch

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    out = {}

    def timed(s, steps, f):
        t = 0.0
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            _, en = s.force_calc(1, f=f)
            t += s.last_time("force")
        return t / steps, en

    for n, forms in ((40, ("fp32",)), (50, ("mlp",))):
        d = tempfile.mkdtemp(prefix=f"mapp_bench_{n}_")
        w = fx.write_workload(d, "dmd", n=n, a=WORKLOAD["a"], sigma=WORKLOAD["sigma"], style="DMD_I")
        s = mb.system_from_workload(w, device=device)
        natms = s.natms
        f64 = torch.zeros((natms, s.x_dim), dtype=torch.float64, device="cuda")
        s.force_calc(1, f=f64)
        t64, en64 = timed(s, 10, f64)
        s.create_2nd_neigh_lst()
        s.c_d_calc()
        mu64 = s.vector("n")
        for form in forms:
            if form == "mlp":
                s.mlp_init(1.8, 5.0, 0.05, 0.20, seed=5)
                par, scal = mlp_source.mlp_state()
                s.mlp_state(params=par, scaling=scal)
                s.set_form(mb.MG_FORM_MLP)
            else:
                s.set_form(mb.MG_FORM_FP32)
            fx_ = torch.zeros_like(f64)
            s.force_calc(1, f=fx_)
            tf, enf = timed(s, 10, fx_)
            rec = {"sites": natms, "ms_per_force_call": tf, "fp64_ms_per_force_call": t64,
                   "site_force_evals_per_s": natms / (tf * 1e-3), "speedup_vs_fp64": t64 / tf,
                   "max_abs_dF_eV_per_A": float((fx_ - f64).abs().max().item()),
                   "abs_dE_per_site_eV": abs(float(enf[0]) - float(en64[0])) / natms}
            if form == "fp32":
                s.create_2nd_neigh_lst()
                s.c_d_calc()
                rec["max_abs_dmu"] = float(np.max(np.abs(s.vector("n") - mu64)))
            else:
                audit, counts = s.mlp_audit()
                rec["audited_rows"] = int(counts[0])
                rec["fallback_rows"] = int(counts[1])
            out[f"{form}_{natms}_sites"] = rec
            s.set_form(mb.MG_FORM_FP64)
        if n == 40:
            # the 256000-site workflow: 200 conjugate-gradient iterations in the
            # precision form (mg_min_cg), then Adams-clock steps of order 2 on
            # the relaxed state (plain form; dt = 1e-3 / rms(c_d))
            s.set_form(mb.MG_FORM_FP32)
            t0 = time.perf_counter()
            r, st = s.min_cg(200, 1e-5, 1e-8, 60, cluster=0)
            wall = time.perf_counter() - t0
            out["cg_fp32_256000_sites"] = {
                "iterations": r["iterations"], "evaluations": r["evaluations"], "stop_code": r["code"],
                "energy": r["energy"], "max_f": r["max_f"], "wall_s": wall, "relax_ms": st["relax_ms"],
                "build_ms": st["build_ms"], "tune_ms": st["tune_ms"],
                "ms_per_evaluation": st["relax_ms"] / max(r["evaluations"], 1),
                "lbfgs_cluster": st["lbfgs_cluster"]}
            s.set_form(mb.MG_FORM_FP64)
            s.create_2nd_neigh_lst()
            s.force_calc(1)
            cd = s.c_d_calc()
            dt = 1e-3 / float(np.sqrt(np.mean(cd * cd)))
            s.clock_adams(2, 1, dt)  # warm-up (first-call allocations)
            t0 = time.perf_counter()
            ra = s.clock_adams(2, 10, dt)
            wall = time.perf_counter() - t0
            out["adams_256000_sites"] = {"order": 2, "steps": 10, "dt": dt, "wall_s": wall,
                                         "ms_per_step": wall * 1e3 / 10, "calc_g_calls": ra["n_calc_g"],
                                         "final_cost_max": float(np.max(ra["err"]))}
            # 100 BDF steps of order at most 2 from 1e-3 tau on the same
            # lattice with the DMD_II force field (with DMD_I the reference's
            # Clock_BDF stalls against the [0, 1] box, see run_bdf)
            d2 = tempfile.mkdtemp(prefix="mapp_bdf256_")
            w2 = fx.write_workload(d2, "dmd", n=40, a=WORKLOAD["a"], sigma=0.0, style="DMD_II", seed=4321)
            s2 = mb.system_from_workload(w2, device=device)
            s2.create_2nd_neigh_lst()
            s2.force_calc(1)
            cd2 = s2.c_d_calc()
            tau2 = 1.0 / float(np.sqrt(np.mean(cd2 * cd2)))
            s2.clock_bdf(2, max_order=2, initial_del_t=1e-3 * tau2)  # warm-up
            s2.close()
            # the median of five runs from the same start (the host steers
            # every solve, so the wall time follows the host's load: single
            # runs of 1.3-1.5 s against 0.56 s were seen on a loaded host)
            walls = []
            for _ in range(5):
                s2 = mb.system_from_workload(w2, device=device)
                t0 = time.perf_counter()
                rb = s2.clock_bdf(100, max_order=2, initial_del_t=1e-3 * tau2)
                walls.append(time.perf_counter() - t0)
                s2.close()
            wall = float(np.median(walls))
            out["bdf2_256000_sites"] = {"style": "DMD_II", "steps": rb["steps"], "initial_del_t": 1e-3 * tau2,
                                        "final_time": rb["t"], "orders_used": np.bincount(rb["order"]).tolist(),
                                        "wall_s": wall, "walls_s": walls, "wall_s_min": min(walls),
                                        "ms_per_step": wall * 1e3 / max(rb["steps"], 1),
                                        "calc_g_calls": rb["n_calc_g"],
                                        "ms_per_calc_g": wall * 1e3 / max(rb["n_calc_g"], 1)}
        s.close()
    return out


def run_single_lbfgs(mb, w, device):
    """Device-resident L-BFGS of the 32000-site system itself (mg_min_lbfgs;
    m = 5, max|f| < 1e-5, energy tolerance 1e-8, 60 halvings, at most 200
    iterations), with the L-BFGS step's cluster size autotuned; beside it the
    cost of one force evaluation through the C ABI with host copies, which a
    host-side minimiser pays per evaluation."""
    s = mb.system_from_workload(w, device=device)
    r, st = s.min_lbfgs(5, 200, 1e-5, 1e-8, 60, cluster=0)
    out = {"sites": s.natms, "relax_ms": st["relax_ms"], "build_ms": st["build_ms"], "tune_ms": st["tune_ms"],
           "iterations": r["iterations"], "evaluations": r["evaluations"],
           "ms_per_evaluation": st["relax_ms"] / max(r["evaluations"], 1), "stop_code": r["code"],
           "max_f": r["max_f"], "energy": r["energy"],
           "launch_shapes": {"bps1": st["bps1"], "bps2": st["bps2"], "lbfgs_threads": st["lbfgs_threads"],
                             "lbfgs_cluster": st["lbfgs_cluster"]}}
    s.close()
    return out


MD_DT = 0.0982269    # 1 fs in the reference's sqrt(amu A^2 / eV) time unit
MD_KB = 8.617333e-5  # eV / K


def run_md(mb, fx, device, steps=1000, ref_steps=300):
    """Nose-Hoover NVT of the FCC 10^3 EAM crystal (4000 atoms, a = 3.615 A,
    sites displaced by sigma = 0.05 A, setfl tables of species A): create_vel
    at 300 K, thermostat period 100 fs, 1000 steps of 1 fs through mg_md_nh,
    timed on the host clock around the call (velocity set-up, the initial
    force, every step, rebuilds and the copies out included); beside it the
    reference's own MD_NH on the same system for ref_steps steps on one core."""
    d = tempfile.mkdtemp(prefix="mapp_md_")
    w = fx.write_workload(d, "eam", n=10)
    period = 100 * MD_DT
    s = mb.system_from_workload(w, device=device)
    s.md_nh(300.0, period, 20, MD_DT, MD_KB, seed=4321)  # warm-up: module load, graph paths
    s.close()
    s = mb.system_from_workload(w, device=device)
    t0 = time.perf_counter()
    r = s.md_nh(300.0, period, steps, MD_DT, MD_KB, seed=4321)
    wall = time.perf_counter() - t0
    n = s.natms
    out = {"atoms": n, "steps": steps, "wall_s": wall, "ms_per_step": wall * 1e3 / steps,
           "atom_steps_per_s": n * steps / wall, "rebuilds": r["rebuilds"], "final_T": r["t"],
           "final_energy": r["energy"],
           "config": "FCC 10^3 EAM (setfl, species A), create_vel 300 K, period 100 fs, dt 1 fs, skin 0.5 A",
           "kernels_per_step": 6, "timing": "host clock around mg_md_nh (set-up, steps, rebuilds, copies out)"}
    s.close()
    from oracle import reference

    if reference.available():
        rr = reference.RefRun(w, workdir=os.path.join(d, "ref"), init=False)
        rr.md(300.0, period, ref_steps, MD_DT, MD_KB, seed=4321)
        meta = rr.run(timeout=1800)["md"]["meta"]
        t_ref = float(meta["time_run"])
        out["cpu_baseline"] = {"value": n * ref_steps / t_ref, "unit": "atom-steps/s", "cores": 1,
                               "kind": "reference",
                               "sample": f"reference MD_NH::run, {ref_steps} steps of the same system, {t_ref:.2f} s"}
        out["speedup_vs_reference_core"] = out["atom_steps_per_s"] / out["cpu_baseline"]["value"]
    return out


def run_adams(mb, w, device, order=2, steps=20, ref_steps=1, with_reference=True):
    """Adams clock of the 32000-site DMD_I system (mg_clock_adams): order 2,
    dt = 1e-3 tau with tau = 1 / rms(c_d) at the start, 20 steps, timed on the
    host clock around the call (crd list, initial force, every calc_g / c_d
    and the scalar read-backs included); beside it the reference's own
    Clock_Adams on the same system for ref_steps steps on one core."""
    s = mb.system_from_workload(w, device=device)
    s.create_2nd_neigh_lst()
    s.force_calc(1)
    cd = s.c_d_calc()
    tau = 1.0 / float(np.sqrt(np.mean(cd * cd)))
    dt = 1e-3 * tau
    s.clock_adams(order, 2, dt)  # warm-up
    s.close()
    # the clock steers every solve from the host, so its wall time follows the
    # host's load: the median of three runs from the same start is reported
    walls = []
    for _ in range(3):
        s = mb.system_from_workload(w, device=device)
        t0 = time.perf_counter()
        r = s.clock_adams(order, steps, dt)
        walls.append(time.perf_counter() - t0)
        n = s.natms
        s.close()
    wall = float(np.median(walls))
    out = {"sites": n, "order": order, "steps": steps, "dt": dt, "tau": tau, "wall_s": wall, "walls_s": walls,
           "ms_per_step": wall * 1e3 / steps, "calc_g_calls": r["n_calc_g"],
           "ms_per_calc_g": wall * 1e3 / max(r["n_calc_g"], 1), "final_cost_max": float(np.max(r["err"])),
           "site_steps_per_s": n * steps / wall,
           "timing": "host clock around mg_clock_adams (crd list, initial force, solves)"}
    s.close()
    from oracle import reference

    if with_reference and reference.available():
        rr = reference.RefRun(w, workdir=tempfile.mkdtemp(prefix="mapp_adams_"), init=False)
        rr.adams(order, ref_steps, dt)
        meta = rr.run(timeout=1800)["adams"]["meta"]
        t_ref = float(meta["time_run"])
        out["cpu_baseline"] = {"value": n * ref_steps / t_ref, "unit": "site-steps/s", "cores": 1, "kind": "reference",
                               "sample": f"reference Clock_Adams::run, {ref_steps} step(s) of the same system "
                                         f"({meta['n_calc_g']} calc_g), {t_ref:.2f} s"}
        out["speedup_vs_reference_core"] = out["site_steps_per_s"] / out["cpu_baseline"]["value"]
    return out


def run_bdf(mb, fx, device, steps=100, ref_steps=5, with_reference=True, cells=20):
    """BDF clock (mg_clock_bdf) of the FCC cells^3 (default 20^3 = 32000-site)
    binary DMD system with the
    DMD_II force field: "clock bdf 100 max_order 2 initial_del_t 1e-3 tau"
    (tau = 1 / rms(c_d) at the start), the reference's own step-size and
    order control, timed on the host clock around the call (crd list,
    initial force, every calc_g and the scalar read-backs included).  DMD_II
    because with DMD_I the reference's own Clock_BDF stops progressing on
    this lattice: its calc_g never refreshes c_d, so the predictor keeps the
    initial rates and drives a site against the [0, 1] box, where its retry
    loop never ends.  Beside it the reference's Clock_BDF for the first
    ref_steps steps on one core, and ours over the same steps."""
    d = tempfile.mkdtemp(prefix="mapp_bdf_")
    w = fx.write_workload(d, "dmd", n=cells, a=WORKLOAD["a"], sigma=0.0, style="DMD_II", seed=4321)
    s = mb.system_from_workload(w, device=device)
    s.create_2nd_neigh_lst()
    s.force_calc(1)
    cd = s.c_d_calc()
    tau = 1.0 / float(np.sqrt(np.mean(cd * cd)))
    opts = dict(max_order=2, initial_del_t=1e-3 * tau)
    s.clock_bdf(3, **opts)  # warm-up
    s.close()
    # the median of five runs from the same start (the host steers every
    # solve, so the wall time follows the host's load)
    walls, walls_s = [], []
    for _ in range(5):
        s = mb.system_from_workload(w, device=device)
        n = s.natms
        t0 = time.perf_counter()
        r = s.clock_bdf(steps, **opts)
        walls.append(time.perf_counter() - t0)
        s.close()
        s = mb.system_from_workload(w, device=device)
        t0 = time.perf_counter()
        rs = s.clock_bdf(ref_steps, **opts)
        walls_s.append(time.perf_counter() - t0)
        s.close()
    wall, wall_s = float(np.median(walls)), float(np.median(walls_s))
    out = {"sites": n, "style": "DMD_II", "max_order": 2, "steps": r["steps"], "initial_del_t": opts["initial_del_t"],
           "tau": tau, "final_time": r["t"], "orders_used": np.bincount(r["order"]).tolist(), "wall_s": wall,
           "ms_per_step": wall * 1e3 / max(r["steps"], 1), "calc_g_calls": r["n_calc_g"],
           "ms_per_calc_g": wall * 1e3 / max(r["n_calc_g"], 1), "site_steps_per_s": n * r["steps"] / wall,
           "walls_s": walls, "wall_s_min": min(walls),
           "first_steps": {"steps": rs["steps"], "wall_s": wall_s, "calc_g_calls": rs["n_calc_g"]},
           "timing": "host clock around mg_clock_bdf (crd list, initial force, solves, step control)"}
    from oracle import reference

    if with_reference and reference.available():
        rr = reference.RefRun(w, workdir=tempfile.mkdtemp(prefix="mapp_bdf_ref_"), init=False)
        rr.bdf(ref_steps, **opts)
        meta = rr.run(timeout=1800)["bdf"]["meta"]
        t_ref = float(meta["time_run"])
        out["cpu_baseline"] = {"value": n * ref_steps / t_ref, "unit": "site-steps/s", "cores": 1, "kind": "reference",
                               "sample": f"reference Clock_BDF::run, the first {ref_steps} steps of the same run "
                                         f"({meta['n_calc_g']} calc_g), {t_ref:.2f} s"}
        out["speedup_vs_reference_core_same_steps"] = t_ref / wall_s
    return out


def run_ours(args):
    import torch

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    import mapp_b200 as mb
    from mapp_b200 import fixtures as fx

    d = tempfile.mkdtemp(prefix=f"mapp_bench_{rank}_")
    w = fx.write_workload(d, "dmd", n=args.cells, a=WORKLOAD["a"], sigma=WORKLOAD["sigma"], style="DMD_I",
                          seed=4321 + rank)
    s = mb.system_from_workload(w, device=local)
    natms = s.natms
    nt = s.nt
    cnt = s.counts()
    f_dev = torch.zeros((natms, s.x_dim), dtype=torch.float64, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    # pairs inside the smeared cut (for the algorithmic FLOP count), from the list itself
    sizes, pairs = s.neighbor_list()
    xo = s.get_x()
    gx, _ = s.ghosts()
    xall = np.concatenate([xo, gx])[:, :3]
    ii = np.repeat(np.arange(natms), sizes)
    rsq = np.sum((xall[ii] - xall[pairs]) ** 2, axis=1)
    mod_rc = 5.0 + 1.224744871391589 / np.sqrt(20.0)
    in_cut = int(np.count_nonzero(rsq < mod_rc * mod_rc))

    form_id = {"fp64": mb.MG_FORM_FP64, "fp32": mb.MG_FORM_FP32, "mlp": mb.MG_FORM_MLP}[args.form]
    if args.form != "fp64":
        args.skip_forms = True
    if args.form == "mlp":
        s.mlp_init(1.8, 5.0, 0.05, 0.20, seed=5)
        s.mlp_train(nsamples=2_000_000, steps=20_000, batch=4096, lr=1e-3, seed=11)
    s.set_form(form_id)
    t_dev = 0.0
    t_ph = [0.0, 0.0, 0.0]
    # nvidia-smi samples every 200 ms and takes a moment to start, so the
    # sampler starts before the warm-up and, after a short timed region, runs
    # on through further (untimed) steps of the same work until it has a few
    # samples under this load
    with Clocks(local) as clk:
        for _ in range(args.warmup):
            s.force_calc(1, f=f_dev)
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        wall0 = time.perf_counter()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            s.force_calc(1, f=f_dev)
            t_dev += s.last_time("force")
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
        t_extra = time.perf_counter()
        while clk.count() < 5 and time.perf_counter() - t_extra < 3.0:
            for _ in range(20):
                flush.zero_()
                s.force_calc(1, f=f_dev)
            torch.cuda.synchronize()
    # the per-kernel times (the roofline's pass 1 among them): the same steps
    # again, with the library's phase events on
    ph = phase_times(s, f_dev, args.steps, flush)
    t_ph = [v * args.steps for v in ph[:3]]
    t_dev_phased = ph[3]
    t_p1 = t_ph[0]
    t_dev = job_max(t_dev, "cuda")
    if ws > 1:
        dist.barrier()
    value = job_rate(natms, args.steps, t_dev * 1e-3, ws)

    if ws > 1:
        # several GPUs: the single-system forms are per-GPU figures; the form
        # that splits across GPUs is the batched one (cells shared out by
        # cost, one graph launch per rank, results gathered on rank 0)
        args.skip_forms = True
    forms = {} if args.skip_forms else run_forms(args, s, mb, natms, f_dev, flush, t_dev)
    if ws > 1:
        forms["batched_sharded"] = run_batched_sharded(mb, fx, local, rank, ws)
    if not args.skip_forms:
        forms["batched"] = run_batched(mb, fx, local)
        forms["single_lbfgs"] = run_single_lbfgs(mb, w, local)
        forms["md_nh"] = run_md(mb, fx, local)
        forms["clock_adams"] = run_adams(mb, w, local)
        forms["clock_bdf"] = run_bdf(mb, fx, local)
        forms["large"] = run_large_forms(mb, fx, local, s)
    s.set_form(form_id)

    # end to end through the C ABI with host buffers, timed with CUDA events on
    # the stream the library runs on (host gaps between the calls included)
    x_host = torch.from_numpy(xo.copy()).pin_memory()
    c_host = torch.from_numpy(np.ascontiguousarray(w["cfg"].c)).pin_memory()
    f_host = torch.zeros((natms, s.x_dim), dtype=torch.float64).pin_memory()
    e2e_stream = torch.cuda.Stream()
    s.set_stream(e2e_stream.cuda_stream)
    # update_x as a MAPP binding calls it (no rebuilt flag asked for: the
    # skin test is read with force_calc's results), and no timing events, as
    # a production caller runs
    s.set_timing(0)
    for _ in range(2):
        s.update_x(x_host, report=False)
        s.update_c(c_host)
        s.force_calc(1, f=f_host)
    torch.cuda.synchronize()
    e2e_steps = max(10, args.steps // 4)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(e2e_stream)
    for _ in range(e2e_steps):
        s.update_x(x_host, report=False)
        s.update_c(c_host)
        s.force_calc(1, f=f_host)
    ev1.record(e2e_stream)
    torch.cuda.synchronize()
    t_e2e = job_max(ev0.elapsed_time(ev1) * 1e-3, "cuda")
    e2e_py = job_rate(natms, e2e_steps, t_e2e, ws)
    _, en_py = s.force_calc(1, f=f_host)
    s.set_timing(1)
    # the same steps from a C++ caller of the C ABI (mapp_b200/client/mapp_e2e.cpp),
    # as MAPP's force loop would make them: set up from the same CFG file and
    # ff_coef arguments, pinned host buffers, events on the library's stream
    e2e_client = run_e2e_client(mb, w, e2e_steps, local) if args.form == "fp64" else None
    t_client = job_max(e2e_client["ms"] * 1e-3 if e2e_client else float("inf"), "cuda")
    if np.isfinite(t_client):
        e2e_value = job_rate(natms, e2e_steps, t_client, ws)
        e2e_path = ("C++ client of the C ABI (mapp_b200/client/mapp_e2e.cpp): mg_atoms_update_x (rebuilt flag not "
                    "asked for, as MAPP's callers) + mg_atoms_update_c + mg_ff_force_calc, pinned host buffers")
    else:
        e2e_value, e2e_client = e2e_py, None
        e2e_path = "mg_atoms_update_x + mg_atoms_update_c + mg_ff_force_calc through ctypes, pinned host buffers"

    # side measurements (list build, energy_calc, c_d_calc, calc_g): the median
    # of five calls after one untimed call (a kernel's first launch in a
    # process also loads its code)
    def side(call, phase):
        call()
        ts = []
        for _ in range(5):
            call()
            ts.append(s.last_time(phase))
        return float(np.median(ts))

    t_list = side(s.rebuild_list, "list")
    t_energy = side(s.energy_calc, "energy")
    s.create_2nd_neigh_lst()
    t_cd = side(s.c_d_calc, "c_d")
    a_zero = np.zeros((natms, nt))
    t_g = side(lambda: s.calc_g(a_zero, 1e-3), "calc_g")

    if rank != 0:
        if ws > 1:
            dist.destroy_process_group()
        return 0

    peaks, peak_kind = measured_peaks()
    p1_ms, emb_ms, p2_ms = (t / args.steps for t in t_ph)
    call_ms = t_dev / args.steps
    f1 = pass1_flops_per_pair(nt, 3) * in_cut
    f2 = pass2_flops_per_pair(nt) * in_cut
    bytes_p1 = PASS1_ALG_BYTES_PER_SITE * natms
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved_gbs = bytes_p1 / (p1_ms * 1e-3) / 1e9
    # DRAM bytes (read + write) of one k_dmd_pass1 launch from the committed ncu
    # capture, per owned site, scaled to this system
    traffic = None
    tf = os.path.join(ROOT, "profiles", "dmd_pass1_traffic.json")
    if os.path.exists(tf) and args.form == "fp64":
        try:
            with open(tf) as fp:
                traffic = json.load(fp)["bytes_per_site"] * natms
        except (OSError, KeyError, ValueError):
            traffic = None
    clocks = clk.summary()
    tflops = lambda fl, ms: fl / (ms * 1e-3) / 1e12
    flop_rules = {"pass1": "nt^2 (10 + 22 nq) flops per half pair inside the smeared cut (304 here)",
                  "pass2": "nt^2 * 25 flops per half pair inside the smeared cut (100 here)",
                  "force_call": "pass1 + pass2 rules (404 per half pair inside the smeared cut here)"}
    if args.form == "fp64":
        peak = measure_fp64_peak()
        peak_note = "measured in this run: cuBLAS DGEMM (torch.matmul float64 4096^3, best of 5); " \
                    "MEASURED_PEAKS.json has no FP64 figure"
        roof = {"bound": "fp64", "kernel": "k_dmd_pass1", "achieved": tflops(f1, p1_ms), "peak": peak,
                "unit": "TFLOP/s", "frac": tflops(f1, p1_ms) / peak, "traffic": traffic,
                "launch_ms": p1_ms, "launch_timing": "CUDA events around the kernel on the library's stream, "
                                                     "in a second loop of the timed steps with phase events on",
                "flops_per_launch": f1, "flops_rule": flop_rules["pass1"],
                "peak_kind": peak_note,
                "pass2": {"kernel": "k_dmd_pass2", "launch_ms": p2_ms, "flops_per_launch": f2,
                          "achieved": tflops(f2, p2_ms), "frac": tflops(f2, p2_ms) / peak,
                          "flops_rule": flop_rules["pass2"]},
                "force_call": {"ms": call_ms, "flops": f1 + f2, "achieved": tflops(f1 + f2, call_ms),
                               "frac": tflops(f1 + f2, call_ms) / peak, "flops_rule": flop_rules["force_call"]},
                "hbm_view": {"achieved_gbs": achieved_gbs, "peak_gbs": hbm, "frac": achieved_gbs / hbm,
                             "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                             "algorithmic_bytes_per_launch": bytes_p1,
                             "algorithmic_bytes_rule": f"{PASS1_ALG_BYTES_PER_SITE} B per owned site "
                                                       "(x, alpha, c read; E written)",
                             "traffic_note": "pass 1 writes the per-pair scratch the reference keeps (21 FP64 "
                                             "values per listed pair); that is most of its DRAM traffic"},
                # what does bind the kernel, from its ncu capture (not measured in this run)
                "binding_resource": {"resource": "L1/TEX data pipe (one wavefront per lane for the knot "
                                                 "and site gathers, about 30 per in-cut pair)",
                                     "utilisation": 0.74, "fp64_pipe": 0.30,
                                     "source": "profiles/k_dmd_pass1_32k.md (ncu --set full, 32000 sites)"}}
    elif args.form == "fp32":
        peak = measure_fp32_peak()
        fB = f1 + f2  # the force pass evaluates the whole smearing and the projection
        roof = {"bound": "fp32", "kernel": "k_dmd32_force", "achieved": tflops(fB, p2_ms), "peak": peak,
                "unit": "TFLOP/s", "frac": tflops(fB, p2_ms) / peak, "traffic": None,
                "launch_ms": p2_ms, "flops_per_launch": fB,
                "flops_rule": "pass1 + pass2 rules: the force pass re-evaluates the smearing with derivatives "
                              "and projects it (404 flops per half pair inside the smeared cut here)",
                "peak_kind": "measured in this run: cuBLAS SGEMM (torch.matmul float32, TF32 off, 8192^3, best of 5)",
                "density_pass": {"kernel": "k_dmd32_dens", "launch_ms": p1_ms},
                "force_call": {"ms": call_ms, "flops": fB, "achieved": tflops(fB, call_ms),
                               "frac": tflops(fB, call_ms) / peak, "flops_rule": flop_rules["force_call"]}}
    else:
        bf16 = float(peaks.get("bf16_tflops", 1590.0))
        _, mlp_counts = s.mlp_audit()
        net_rows = nt * nt * in_cut - int(mlp_counts[1])
        fm = MLP_FLOPS_PER_ROW * net_rows
        roof = {"bound": "tensor", "kernel": "k_mlp_rows .. k_mlp_densities (the learned pass 1)",
                "achieved": tflops(fm, p1_ms), "peak": bf16,
                "unit": "TFLOP/s", "frac": tflops(fm, p1_ms) / bf16, "traffic": None, "launch_ms": p1_ms,
                "flops_per_launch": fm, "network_rows": net_rows,
                "flops_rule": "network flops per row (17664) x rows inside the training box (nt^2 rows per half "
                              "pair inside the smeared cut, less the quadrature-fallback rows the call counted)",
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json bf16_tflops)"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_dev / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp64": "f64", "fp32": "f32", "mlp": "bf16"}[args.form],
        "data": "synthetic (seeded lattice, alpha and c; random tables of the named potentials)",
        "form": {"fp64": "plain FP64", "fp32": "precision (FP32)", "mlp": "learned (BF16 MLP)"}[args.form],
        "config": workload_config(args),
        "workload_counts": {"pairs": cnt["npairs"], "pairs_in_smeared_cut": in_cut, "ghosts": cnt["nph"]},
        "roofline": roof,
        "e2e": {"value": e2e_value, "unit": UNIT,
                # down: f, then the 8 totals and 8 status words in one copy
                "h2d_bytes_per_step": natms * (s.x_dim + nt) * 8, "d2h_bytes_per_step": natms * s.x_dim * 8 + 96,
                "steps": e2e_steps, "path": e2e_path,
                "python_ctypes": {"value": e2e_py, "path": "the same calls from Python through ctypes"},
                "client_energy_rel_diff": (abs(e2e_client["energy"] - float(en_py[0])) / abs(float(en_py[0]))
                                           if e2e_client else None)},
        "forms": forms,
        # library kernels per force call: plain pass 1, embedding, pass 2,
        # reduction; precision prep, density, embedding, force, merge,
        # reduction; learned rows, fallback, network, audit, densities,
        # embedding, pass 2, reduction
        "gpu_launches": {"fp64": 4, "fp32": 6, "mlp": 8}[args.form] * args.steps,
        "phases_ms": {"force": t_dev / args.steps, "force.pass1": p1_ms, "force.embed": emb_ms,
                      "force.pass2": p2_ms, "force_with_phase_events": t_dev_phased,
                      "phase_note": "per-kernel times from a second loop of the same steps with the library's "
                                    "phase events on (they cost the call a few us, so the timed loop runs without)",
                      "list_rebuild": t_list,
                      "energy_calc": t_energy, "c_d_calc": t_cd, "calc_g": t_g},
        "wall_s": wall,
        "clocks": clocks,
    }
    if not args.no_cpu and ws == 1:
        reps = args.cpu_reps or 3
        procs = os.cpu_count() or 1
        r = cpu_reference(w, natms, reps, procs)
        if r is not None:
            line["cpu_baseline"] = {"value": r["value"], "unit": UNIT, "cores": procs, "kind": "reference",
                                    "sample": f"{procs} concurrent single-rank reference processes x {reps} "
                                              f"force_calc calls of the {natms}-site system ({cpu_model()}), "
                                              f"{r['wall']:.1f} s"}
    print(json.dumps(line))
    if ws > 1:
        dist.destroy_process_group()
    return 0


def run_eam(args):
    """EAM force_calc of the Nose-Hoover crystal's potential (species A setfl
    tables) on FCC n^3 atoms, a = 3.615 A, sites displaced by 0.05 A: the MD
    loop's force path timed alone (CUDA events of the library), one JSON line.
    A profiling entry; the default run reports the MD loop itself."""
    import torch
    import mapp_b200 as mb
    from mapp_b200 import fixtures as fx

    w = fx.write_workload(tempfile.mkdtemp(prefix="mapp_eam_"), "eam", n=args.eam_cells)
    s = mb.system_from_workload(w)
    f = torch.zeros((s.natms, 3), dtype=torch.float64, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        s.force_calc(1, f=f)
    t = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        s.force_calc(1, f=f)
        t += s.last_time("force")
    ms = t / args.steps
    print(json.dumps({"metric": "EAM atom-force evals/s", "value": s.natms / (ms * 1e-3), "unit": "atom-force evals/s",
                      "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup, "dtype": "f64",
                      "config": {"workload": f"FCC {args.eam_cells}^3 EAM (species A setfl)", "atoms": s.natms,
                                 "pairs": s.counts()["npairs"]}}))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.eam_cells > 0:
        return run_eam(args)
    if args.clock:
        import torch

        import mapp_b200 as mb
        from mapp_b200 import fixtures as fx

        torch.cuda.set_device(0)
        if args.clock == "bdf":
            out = run_bdf(mb, fx, 0, with_reference=False, cells=args.cells)
        else:
            w = fx.write_workload(tempfile.mkdtemp(prefix="mapp_adams_w_"), "dmd", n=WORKLOAD["n"], a=WORKLOAD["a"],
                                  sigma=WORKLOAD["sigma"], style="DMD_I", seed=4321)
            out = run_adams(mb, w, 0, with_reference=False)
        print(json.dumps({"clock": args.clock, **out}))
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
