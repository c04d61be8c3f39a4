#!/usr/bin/env python
"""Benchmark: trapezoidal steps/s on the 128x128x32 holed film (one B200).

Workload (the precision-form configuration): Nx=Ny=128, Nz=32 cells,
h=0.5, kappa=2, Bz=0.5 switched on for the whole run, a centred square hole
with vertices (24,24)-(40,40) (32x32 nodes through all 33 planes), seeded
psi0 = 1 + 0.01 (N + iN) outside the hole, phi0 = 0; dt = 0.1, Newton
tol_f = 1e-8, tol_dx = 1e-3, GCR tol 1e-6, eps_mf = 1e-4.  A "step" is one
accepted trapezoidal step (predictor, Newton iterations with their GCR solves).

Arms:
  --impl ours       the device stepper (default: mixed precision, FP32 Krylov
                    vectors / FP64 state and reductions); also times the FP64
                    stepper on the same steps and reports the |psi|^2 error.
  --impl reference  the CPU oracle (numpy restatement of the reference
                    algorithm) on the host cores, same workload and metric.

One JSON line on rank 0.  Under torchrun (N > 1) every rank runs an
independent replica (the stepper does not shard); value = N * K / max time.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "trapezoidal steps/s @128²×32: mixed-FP32 vs FP64 at 1e-6 rel err; % HBM peak"
WORKLOAD = dict(Nx=128, Ny=128, Nz=32, h=0.5, kappa=2.0, Bz=0.5, hole=[(24, 24), (40, 24), (40, 40), (24, 40)],
                dt=0.1, tol_f=1e-8, tol_dx=1e-3, tol_gcr=1e-6, eps_mf=1e-4, seed=3, t_stop=50.0)
WORKLOAD_NAME = ("trapezoidal step, 128x128x32-cell film (499,999 interior nodes), 32x32-node hole through "
                 "all planes, h=0.5, kappa=2, Bz=0.5, dt=0.1, Newton tol_f 1e-8 / tol_dx 1e-3, GCR tol 1e-6")
HBM_FALLBACK_GBS = 6650.0
WORKLOAD_N_INTERIOR = 127 * 127 * 31
# DRAM bytes per algorithmic byte of the GMRES step graph on the 128x128x32
# workload at the default preconditioner degree (8), from a graph-level ncu
# capture (dram__bytes_read.sum + dram__bytes_write.sum) of the timed 2-step
# launch of `bench.py --steps 2 --warmup 3 --no-fp64 --no-e2e
# --no-cpu-baseline --no-forms`: 0.909 GB read + 1.541 GB written = 2.450 GB
# against 8.082 GB algorithmic.  The stencil launches' vectors stay in L2;
# the projections read most of the basis from DRAM.
DRAM_PER_ALG_BYTE = 0.2907
DRAM_RATIO_DEGREE = 10


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--kmax", type=int, default=64)
    ap.add_argument("--krylov", choices=["gmres", "gcr"], default="gmres")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the other forms (trilayer, batched, differentiation) after the headline line")
    ap.add_argument("--cpu-budget-s", type=float, default=150.0)
    ap.add_argument("--form", choices=["precision", "adjoint", "batched", "trilayer"], default="precision",
                    help="adjoint: gradients of the 64x64x16 differentiation workload; batched: instance-steps/s "
                         "of 64 uneven instances stepped together against looping them (--steps per instance); "
                         "trilayer: the 256x256x64 S/I/S stack, mixed against FP64")
    ap.add_argument("--adj-smax", type=float, default=ADJ["s_max"],
                    help="upper end of the suppression field s(x) of the differentiation workload")
    ap.add_argument("--probe-no-fill", action="store_true",
                    help="--arnoldi-probe without the two filling steps (no graph launch in the process, "
                         "so ncu can replay the probe's kernels; the basis then holds zeros)")
    ap.add_argument("--arnoldi-probe", type=int, default=None, metavar="J",
                    help="diagnostic: time the three Arnoldi-step kernels standalone at basis index J and exit")
    ap.add_argument("--kernel-timers", action="store_true",
                    help="per-kernel device timers of the step graph (adds a little overhead; not a headline run)")
    return ap.parse_args()


def build_device():
    import nanowire_tdgl_b200 as tb
    w = WORKLOAD
    p = tb.SimulationParameters(Nx=w["Nx"], Ny=w["Ny"], Nz=w["Nz"], hx=w["h"], hy=w["h"], hz=w["h"],
                                kappa=w["kappa"])
    dev = tb.Device(p, applied_field=tb.AppliedField(Bz=w["Bz"], t_on_fraction=1.0))
    dev.add_hole(w["hole"])
    rng = np.random.default_rng(w["seed"])
    x0 = dev.initial_state()
    n = p.n_interior
    x0.psi[:] += 0.01 * (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * dev.material.interior_sc_mask
    return dev, x0.data.copy()


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            v = json.load(fh).get("hbm_gbs")
        if v:
            return float(v), "measured"
    except (OSError, ValueError):
        pass
    return HBM_FALLBACK_GBS, "fallback"


# ---------------------------------------------------------------------------
# algorithmic bytes (per-stage compulsory traffic, stage counts from the device)
# ---------------------------------------------------------------------------

def algorithmic_bytes(n_int: int, precision: str, st: dict, poly_deg: int = 0) -> float:
    """Compulsory HBM bytes of the counted work.

    S64 = 40 B/node (psi complex + 3 real links, FP64 state), SK = bytes/node
    of the Krylov vectors (20 B FP32 in the mixed form, 40 B FP64), F = 1 B/node
    of flags.  Per stage:
      RHS f(x) (predictor, Newton residual)      2 S64 + F
      Jacobian product and A p formation         3 SK + F
      Gram-Schmidt + alpha/x/r updates, solve of m iterations:
                                                  sum_k (2(k-1) + 8) SK = (m^2 + 7 m) SK
      Newton residual, norms, x += dx            7 S64 per Newton iteration
    This is the per-stage model of the reference's GCR form.  The GMRES form
    run here moves, per solve of m iterations, sum_{j=0..m-1} (2 j + 7) SK
    (orthogonalisation j + 2 vectors, product 3, projections j + 2) plus the
    last step's orthogonalisation (its products are skipped once its stop
    check has ended the solve), within a few percent of the model at m ~ 25.
    With the polynomial preconditioner of degree d, every Arnoldi column takes
    d more stencil launches (counted in jvp_evals, 3 SK + F each) that also
    read the vector they precondition (+SK each); the last of them keeps
    p(A) U_j as the preconditioned basis vector the Newton correction combines
    (in place of the basis vector itself, so the update's traffic is
    unchanged).
    """
    S64 = 40.0 * n_int
    SK = (20.0 if precision == "mixed" else 40.0) * n_int
    F = 1.0 * n_int
    poly = poly_deg * st["krylov_iters"] * SK
    return (st["rhs_evals"] * (2 * S64 + F) + st["jvp_evals"] * (3 * SK + F)
            + (st["krylov_sq"] + 7 * st["krylov_iters"]) * SK + 7 * S64 * st["newton_iters"] + poly)


def graph_launches(st: dict, jvp: str, poly_deg: int = 0) -> int:
    """Kernel launches of the step graph: 7 per step attempt, 4 per Newton
    iteration, and per Krylov solve of m iterations either 4 (m + 1)
    (orthogonalisation, stop check, product, projections; analytic products;
    the last step's product and projections return at once) or 5 m
    (finite-difference products); with the polynomial preconditioner of
    degree d, d more per Arnoldi step."""
    base = 7 * (st["steps"] + st["rejections"]) + 4 * st["newton_iters"]
    if jvp == "analytic":
        return base + (4 + poly_deg) * (st["krylov_iters"] + st["newton_iters"])
    return base + 5 * st["krylov_iters"]


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class Clocks:
    QUERY = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self, uuid: str | None):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as fh:
            for line in fh:
                f = [x.strip() for x in line.split(",")]
                if len(f) < 11:
                    continue
                if uuid and uuid not in f[1]:
                    continue
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return None
        def num(v):
            try:
                return float(v)
            except ValueError:
                return None
        load = [r for r in rows if (num(r[5]) or 0) > 0] or rows
        sm = [num(r[2]) for r in load if num(r[2]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in load:
            for nm, v in zip(names, r[7:11]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": num(load[0][3]),
                "reasons": sorted(reasons), "samples": len(rows), "samples_under_load": len(load)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def max_over_ranks(v: float, dist: bool, device) -> float:
    """The largest of every rank's v (the job's time is its slowest
    replica's); v itself on one process."""
    if not dist:
        return float(v)
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, world: int, max_ms: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time."""
    return world * units_per_rank / (max_ms / 1e3)


def device_run(g, x0, opts, fld, warmup, steps, dist):
    import torch
    x = g.pack(x0)
    t, cur = 0.0, WORKLOAD["dt"]
    if warmup > 0:
        rc, t, cur, _ = g.trap_run(x, t, cur, warmup, opts, fld)
        if rc != 0:
            raise RuntimeError(f"warm-up failed with status {rc}")
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    rc, t, cur, st = g.trap_run(x, t, cur, steps, opts, fld)
    e1.record()
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    if rc != 0 or st["steps"] != steps:
        raise RuntimeError(f"timed run failed: status {rc}, {st['steps']} of {steps} steps")
    return x, e0.elapsed_time(e1), st


def run_ours(a, rank, world):
    import torch
    import nanowire_tdgl_b200 as tb
    from nanowire_tdgl_b200 import _lib as L
    from nanowire_tdgl_b200.engine import grid_for

    dist = world > 1
    dev, x0 = build_device()
    p, w = dev.params, WORKLOAD
    n_int = p.n_interior

    def make(prec, jvp):
        g = grid_for(p, dev.idx, dev.material, prec, a.kmax, a.krylov)
        opts = L.TrapOpts(w["t_stop"], w["dt"], 1e-8, w["tol_f"], w["tol_dx"], w["tol_gcr"], w["eps_mf"], 20, 0, 1,
                          L.TDGL_JVP_ANALYTIC if jvp == "analytic" else L.TDGL_JVP_FD)
        fld = L.Field(0.0, 0.0, w["Bz"], 1.0, 0.5, w["t_stop"], 0, 0)
        return g, opts, fld

    jvp = "analytic" if a.precision == "mixed" else "fd"
    if a.kernel_timers:
        os.environ["TDGL_PROFILE"] = "1"    # read when the solver workspace is created
    g, opts, fld = make(a.precision, jvp)
    clocks = Clocks()
    clocks.start()
    x, ms, st = device_run(g, x0, opts, fld, a.warmup, a.steps, dist)
    timers = g.kernel_timers() if a.kernel_timers else None
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(0).uuid)
    except Exception:
        pass
    clk = clocks.stop(uuid)
    ms_max = max_over_ranks(ms, dist, "cuda")
    value = job_rate(a.steps, world, ms_max)

    peak, peak_kind = measured_peak()
    poly_deg = g.poly_degree if (jvp == "analytic" and a.krylov == "gmres") else 0
    alg = algorithmic_bytes(n_int, a.precision, st, poly_deg)
    achieved = alg / (ms / 1e3) / 1e9
    # DRAM bytes per algorithmic byte of the GMRES step graph, measured with ncu
    # (graph-level dram__bytes_read.sum + dram__bytes_write.sum) on a 2-step
    # launch of this workload in mixed precision at the default preconditioner
    # degree; traffic follows the Krylov counters, so it is scaled by this
    # run's algorithmic bytes (reported only at that degree).
    traffic = (DRAM_PER_ALG_BYTE * alg
               if (a.precision == "mixed" and a.krylov == "gmres" and poly_deg == DRAM_RATIO_DEGREE) else None)
    traffic_note = (f"{DRAM_PER_ALG_BYTE} x the algorithmic bytes: the DRAM/algorithmic ratio of a graph-level ncu "
                    "capture of this workload's timed launch at this configuration" if traffic is not None else
                    f"not captured at this configuration (the ratio {DRAM_PER_ALG_BYTE} is for mixed precision, "
                    f"GMRES, preconditioner degree {DRAM_RATIO_DEGREE})")
    out = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 Krylov / f64 state" if a.precision == "mixed" else "f64",
        "data": "synthetic (seeded psi0 noise, phi0 = 0; no dataset involved)",
        "config": {"workload": WORKLOAD_NAME, "precision": a.precision, "jvp": jvp, "krylov": a.krylov,
                   "preconditioner": f"Chebyshev polynomial, degree {poly_deg}" if poly_deg else "none",
                   "krylov_stop": ("tol_gcr relative, or once ||r||_2 <= 0.1 tol_f (forcing term; the Newton "
                                   "test is unchanged)"
                                   if (jvp == "analytic" and a.krylov == "gmres"
                                       and os.environ.get("TDGL_FORCING", "1") != "0") else "tol_gcr relative"),
                   "n_interior": n_int,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": ("inputs larger than L2: each step touches ~0.3 GB (FP64 state, iterate, gamma and f, "
                          "their full-grid copies, the FP32 linearisation copy, Krylov basis and preconditioner "
                          "buffers) against the 126 MB L2; no flush between steps")},
        "node_updates_per_s": value * n_int,
        "gpu_launches": graph_launches(st, jvp, poly_deg) if a.krylov == "gmres" else 1,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_note": traffic_note, "peak_kind": peak_kind,
                     "limiter": ("the roofline is HBM (streaming stencils, no contraction), but the preconditioned "
                                 "step's working set stays mostly in L2 (DRAM traffic ~0.29 x the algorithmic "
                                 "bytes) and the step is bound by the tangent-linear stencil launches, which are "
                                 "latency- and issue-bound (~455 instructions per node at ~42% issue-active with 16 "
                                 "warps per SM; the polynomial steps and products take ~2/3 of the step)"),
                     "algorithmic_bytes_per_launch": alg,
                     "kernel": ("trapezoidal step graph (kg_* kernels under conditional WHILE nodes), one graph "
                                "launch for the K timed steps" if a.krylov == "gmres" else
                                "k_stepper (persistent cooperative kernel, one launch)")},
        "counters": {k: st[k] for k in ("newton_iters", "krylov_iters", "krylov_sq", "rhs_evals", "jvp_evals",
                                        "rejections", "max_krylov")},
        "clocks": clk,
    }
    if timers is not None:
        tot = sum(v["ms"] for v in timers.values()) or 1.0
        out["kernel_timers"] = {k: dict(v, share=v["ms"] / tot, ms_per_step=v["ms"] / a.steps)
                                for k, v in timers.items() if v["launches"]}
        out["kernel_timers_note"] = ("device global-timer spans (first block start to last block end) of the "
                                     "warm-up and timed launches; one-block control kernels and launch gaps "
                                     "not included")
    # FP64 stepper on the same steps, and the |psi|^2 error of this run against it
    if not a.no_fp64 and a.precision == "mixed":
        res = {}
        for mode in ("fd", "analytic"):
            g64, o64, f64 = make("fp64", mode)
            x64, ms64, st64 = device_run(g64, x0, o64, f64, a.warmup, a.steps, dist)
            res[mode] = (x64, ms64, st64, g64)
        x64, ms64, st64, g64 = res["fd"]
        psi_m = g.unpack(x)[:n_int]
        psi_d = g64.unpack(x64)[:n_int]
        p2m, p2d = psi_m.abs() ** 2, psi_d.abs() ** 2
        rel = float(torch.linalg.vector_norm(p2m - p2d) / torch.linalg.vector_norm(p2d))
        out["fp64"] = {mode: {"value": a.steps / (r[1] / 1e3), "ms_per_step": r[1] / a.steps,
                              "newton_iters": r[2]["newton_iters"], "krylov_iters": r[2]["krylov_iters"]}
                       for mode, r in res.items()}
        out["speedup_vs_fp64"] = {mode: out["value"] / world / v["value"] for mode, v in out["fp64"].items()}
        out["rel_l2_psi2_vs_fp64"] = rel
        out["max_abs_psi2_vs_fp64"] = float((p2m - p2d).abs().max())
    # the state after step 1 from the seeded state (t = 0), for the comparison
    # with the oracle's step 1 (computed by the CPU-baseline leg)
    x1 = g.pack(x0)
    rc, _, _, _ = g.trap_run(x1, 0.0, w["dt"], 1, opts, fld)
    if rc == 0:
        out["_x1"] = g.unpack(x1).cpu().numpy()
    # end to end through the public API: host numpy state in, every step's state back to the host
    if not a.no_e2e:
        sched = tb.FieldSchedule(dev.applied_field, p, dev.idx, w["t_stop"])
        kw = dict(newton_tol_f=w["tol_f"], newton_tol_dx=w["tol_dx"], tol_gcr=w["tol_gcr"], eps_mf=w["eps_mf"],
                  save_every=1, progress=False, material=dev.material, precision=a.precision, kmax=a.kmax,
                  krylov=a.krylov)
        # warm-up call: the same W steps as the device run, through the API; the
        # timed call then runs the same K steps from its final host state
        tw, hw = tb.trapezoidal(x0, p, dev.idx, sched, 0.0, a.warmup * w["dt"], w["dt"], **kw)
        xw, t_w = np.ascontiguousarray(hw[:, -1]), float(tw[-1])
        torch.cuda.synchronize()
        if dist:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        times, hist = tb.trapezoidal(xw, p, dev.idx, sched, t_w, t_w + a.steps * w["dt"], w["dt"], **kw)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        el = max_over_ranks(el, dist, "cuda")
        nsteps = len(times) - 1
        sbytes = p.n_state * 16
        out["e2e"] = {"value": world * nsteps / el, "unit": "steps/s", "h2d_bytes_per_step": sbytes / nsteps,
                      "d2h_bytes_per_step": sbytes * (nsteps + 1) / nsteps,
                      "call": "nanowire_tdgl_b200.trapezoidal(x numpy, ..., save_every=1) over the same K steps "
                              "as the device run (after the same W warm-up steps through the API): host state "
                              "in, every step's state back to host memory"}
    return out


def cpu_oracle_steps(max_steps: int, budget_s: float, threads: int, want_state: bool = False):
    """Time the oracle's trapezoidal steps on the host (bounded by budget_s);
    with want_state, also return the state after the first step."""
    from threadpoolctl import threadpool_limits
    from oracle import tdgl_oracle as orc
    dev, x0 = build_device()
    w = WORKLOAD
    g = orc.make_grid(dev.params, dev.idx, dev.material)
    fld = orc.field_schedule(Bz=w["Bz"], t_on_fraction=1.0, t_stop=w["t_stop"])
    X = x0
    t = 0.0
    done = 0
    first = None
    t0 = time.perf_counter()
    with threadpool_limits(limits=threads):
        while done < max_steps:
            times, hist = orc.trapezoidal(X, g, fld, t, w["t_stop"], w["dt"], newton_tol_f=w["tol_f"],
                                          newton_tol_dx=w["tol_dx"], tol_gcr=w["tol_gcr"], eps_mf=w["eps_mf"],
                                          max_steps=1)
            X, t = hist[:, -1], times[-1]
            done += 1
            if done == 1:
                first = X.copy()
            if time.perf_counter() - t0 > budget_s:
                break
    el = time.perf_counter() - t0
    if want_state:
        return done, el, first
    return done, el


def run_reference(a, rank, world):
    if rank != 0:
        return None
    # The path is sequential numpy / scipy work: more BLAS threads only slow its
    # long vector updates (measured 0.024 steps/s on 16 threads against 0.045 on
    # one), so it runs on its fastest setting, one thread.
    cores = 1
    done, el = cpu_oracle_steps(a.steps, a.cpu_budget_s, cores)
    val = done / el
    sample = (f"{done} of {a.steps} requested trapezoidal steps from the seeded state (wall budget "
              f"{a.cpu_budget_s:.0f} s), numpy oracle, 1 thread (its fastest), no warm-up steps")
    return {"metric": METRIC, "impl": "reference", "value": val, "unit": "steps/s", "n_gpus": world,
            "steps": done, "warmup": 0, "ms_per_step": 1e3 * el / max(done, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, "precision": "fp64", "jvp": "fd"},
            "cpu_baseline": {"value": val, "unit": "steps/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def arnoldi_probe(a):
    """Standalone launches of the Arnoldi-step kernels at basis index
    a.arnoldi_probe on the workload's context, after two steps that fill the
    basis: the graph's kernels together, then each kernel alone
    (orthogonalisation, product, projections, fused product and projections,
    the polynomial preconditioner's steps), then the Newton-stage kernels
    (predictor, Newton residual, Newton update over J basis vectors, which
    overwrite the iterate); prints their times."""
    import torch
    from nanowire_tdgl_b200 import _lib as L
    from nanowire_tdgl_b200.engine import grid_for, stream_handle
    dev, x0 = build_device()
    w = WORKLOAD
    g = grid_for(dev.params, dev.idx, dev.material, a.precision, a.kmax, "gmres")
    opts = L.TrapOpts(w["t_stop"], w["dt"], 1e-8, w["tol_f"], w["tol_dx"], w["tol_gcr"], w["eps_mf"], 20, 0, 1,
                      L.TDGL_JVP_ANALYTIC)
    fld = L.Field(0.0, 0.0, w["Bz"], 1.0, 0.5, w["t_stop"], 0, 0)
    x = g.pack(x0)
    if not a.probe_no_fill:
        rc, t, cur, st = g.trap_run(x, 0.0, w["dt"], 2, opts, fld)
        if rc != 0:
            raise RuntimeError(f"filling steps failed with status {rc}")
    j = a.arnoldi_probe
    reps = max(a.steps, 1)
    res = {}
    deg = g.poly_degree
    for name, mask in (("graph", 0), ("orthogonalisation", 1), ("product", 2), ("projections", 4),
                       ("product_and_projections", 8), ("polynomial_steps", 16), ("predict", 32),
                       ("newton_residual", 64), ("newton_update", 128)):
        if mask == 16 and deg == 0:
            continue
        L.check(g.lib.tdgl_arnoldi_probe(g.handle, j, 2, mask, stream_handle()), "tdgl_arnoldi_probe")
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        L.check(g.lib.tdgl_arnoldi_probe(g.handle, j, reps, mask, stream_handle()), "tdgl_arnoldi_probe")
        e1.record()
        torch.cuda.synchronize()
        res[name] = e0.elapsed_time(e1) * 1e3 / reps
    vec = dev.params.n_interior * (20 if a.precision == "mixed" else 40)
    alg = (2 * j + 7 + 4 * deg) * vec
    print(json.dumps({"arnoldi_probe": j, "precision": a.precision, "poly_degree": deg, "us_per_launch": res,
                      "algorithmic_bytes": alg, "achieved_gbs_graph": alg / (res["graph"] * 1e-6) / 1e9,
                      "note": "graph kernels together: orthogonalisation (j+2 vectors), polynomial steps (4 each: "
                              "input, direction, output, state), product (3), projections (j+2); "
                              "polynomial_steps = all deg steps of one Arnoldi step; vector = n_interior x 20 B "
                              "(FP32)"}))
    return 0


ADJ = dict(Nx=64, Ny=64, Nz=16, h=0.5, kappa=2.0, Bz=0.4, dt=0.1, n_steps=400, checkpoint=50, seed=5,
           box=(24, 40, 24, 40, 0, 17), s_max=1.0)


def adjoint_workload(s_max: float = ADJ["s_max"]):
    """The differentiation workload: 64x64x16 film, kappa 2, Bz 0.4, a smooth
    seeded suppression field s(x) in [0, s_max] (sc = 1 - s; the configured
    range is [0, 1]; with the reference's -(1 - sc) psi / 0.1 relaxation, s
    above ~0.1 drives psi towards zero there), seeded psi0."""
    import nanowire_tdgl_b200 as tb
    w = ADJ
    p = tb.SimulationParameters(Nx=w["Nx"], Ny=w["Ny"], Nz=w["Nz"], hx=w["h"], hy=w["h"], hz=w["h"],
                                kappa=w["kappa"])
    idx = tb.construct_indices(p)
    rng = np.random.default_rng(w["seed"])
    z = rng.standard_normal((w["Nz"] + 1, w["Ny"] + 1, w["Nx"] + 1))
    for _ in range(6):                        # smooth: repeated 3-point averages along each axis
        for ax in range(3):
            z = (np.roll(z, 1, ax) + z + np.roll(z, -1, ax)) / 3.0
    s_full = s_max * (z - z.min()) / (z.max() - z.min())
    sc_full = (1.0 - s_full).reshape(-1)
    def material(kappa=w["kappa"]):
        return tb.MaterialMap(kappa=np.full(p.dim_x, kappa), sc_mask=sc_full.copy(),
                              interior_sc_mask=sc_full[np.asarray(idx.interior_to_full)].copy())
    n = p.n_interior
    x0 = np.zeros(p.n_state, dtype=np.complex128)
    x0[:n] = (1.0 + 0.01 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))) * material().interior_sc_mask
    return p, idx, material, x0


def run_adjoint(a, s_max: float = ADJ["s_max"]):
    """Gradient of mean |psi|^2 over the centred box after 400 steps with
    respect to s(x), Bz and kappa; FP32 Krylov forward (mixed) with the FP64
    adjoint, timed; central differences (eps 1e-4) of a tight FP64 forward
    check the Bz and kappa entries of a tight FP64 gradient."""
    import torch
    import nanowire_tdgl_b200 as tb
    w = ADJ
    p, idx, material, x0 = adjoint_workload(s_max)
    t_stop = w["n_steps"] * w["dt"]
    loss = tb.box_mean_psi2(p, w["box"])
    kw = dict(material=material(), B=(0.0, 0.0, w["Bz"]), checkpoint_every=w["checkpoint"])
    tb.trapezoidal_gradient(x0, p, idx, 0.0, 2 * w["dt"], w["dt"], loss, precision="mixed", **kw)   # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = tb.trapezoidal_gradient(x0, p, idx, 0.0, t_stop, w["dt"], loss, precision="mixed",
                                  newton_tol_f=1e-8, newton_tol_dx=1e-3, tol_gcr=1e-6, **kw)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    tight = dict(newton_tol_f=1e-12, newton_tol_dx=1e-10, tol_gcr=1e-11, newton_max_iter=30, kmax=128,
                 adjoint_tol=1e-11)
    ref = tb.trapezoidal_gradient(x0, p, idx, 0.0, t_stop, w["dt"], loss, precision="fp64", **kw, **tight)
    eps = 1e-4
    def L(kappa=w["kappa"], bz=w["Bz"]):
        kk = dict(kw, material=material(kappa), B=(0.0, 0.0, bz))
        pp = p if kappa == w["kappa"] else tb.SimulationParameters(Nx=w["Nx"], Ny=w["Ny"], Nz=w["Nz"], hx=w["h"],
                                                                    hy=w["h"], hz=w["h"], kappa=kappa)
        return tb.trapezoidal_gradient(x0, pp, idx, 0.0, t_stop, w["dt"], loss, precision="fp64", backward=False,
                                       **kk, **tight)["loss"]
    fd_bz = (L(bz=w["Bz"] + eps) - L(bz=w["Bz"] - eps)) / (2 * eps)
    fd_k = (L(kappa=w["kappa"] + eps) - L(kappa=w["kappa"] - eps)) / (2 * eps)
    gs = res["grad_sc"].cpu().numpy()
    return {"form": "adjoint", "workload": "64x64x16 film (59,535 interior nodes), kappa 2, Bz 0.4, smooth s(x) in "
                                           f"[0, {s_max:g}], loss mean |psi|^2 over the centred 16x16x16 box after "
                                           "400 steps dt 0.1, checkpoints every 50",
            "seconds": el, "steps": res["steps"], "adjoint_gmres_iters": res["adjoint_iters"],
            "loss": res["loss"], "grad_Bz": float(res["grad_B"][2]), "grad_kappa": res["grad_kappa"],
            "grad_s_norm": float(np.linalg.norm(gs)),
            "fp64_grad_Bz": float(ref["grad_B"][2]), "fp64_grad_kappa": ref["grad_kappa"],
            "fd_grad_Bz": fd_bz, "fd_grad_kappa": fd_k,
            "rel_err_Bz_vs_fd": abs(float(ref["grad_B"][2]) - fd_bz) / abs(fd_bz),
            "rel_err_kappa_vs_fd": abs(ref["grad_kappa"] - fd_k) / abs(fd_k),
            "rel_err_mixed_vs_fp64_Bz": abs(float(res["grad_B"][2]) - float(ref["grad_B"][2]))
                                        / abs(float(ref["grad_B"][2]))}


BATCH = dict(n=64, seed=11, nxy=(32, 48, 64, 96), nz=(4, 8, 16), h=0.5, kappa=(1.5, 4.0), Bz=(0.1, 1.0),
             holes=(0, 3), side=(4, 16), dt=0.1)


def batched_workload():
    """64 seeded instances: Nx, Ny from {32, 48, 64, 96}, Nz from {4, 8, 16}
    cells, h 0.5, kappa ~ U[1.5, 4], Bz ~ U[0.1, 1], 0-3 rectangular holes of
    side 4-16 nodes (through all planes) at seeded positions at least 2 nodes
    inside the edges, psi0 = 1 + 0.01 (N + iN) outside the holes, phi0 = 0."""
    import nanowire_tdgl_b200 as tb
    w = BATCH
    rng = np.random.default_rng(w["seed"])
    devs, xs, desc = [], [], []
    h = w["h"]
    for _ in range(w["n"]):
        Nx, Ny = (int(v) for v in rng.choice(w["nxy"], 2))
        Nz = int(rng.choice(w["nz"]))
        kappa = float(rng.uniform(*w["kappa"]))
        bz = float(rng.uniform(*w["Bz"]))
        p = tb.SimulationParameters(Nx=Nx, Ny=Ny, Nz=Nz, hx=h, hy=h, hz=h, kappa=kappa)
        d = tb.Device(p, applied_field=tb.AppliedField(Bz=bz, t_on_fraction=1.0))
        nh = int(rng.integers(w["holes"][0], w["holes"][1] + 1))
        for _ in range(nh):
            sx, sy = (int(v) for v in rng.integers(w["side"][0], w["side"][1] + 1, 2))
            i0 = int(rng.integers(2, Nx - 2 - sx + 1))
            j0 = int(rng.integers(2, Ny - 2 - sy + 1))
            d.add_hole([(h * i0, h * j0), (h * (i0 + sx), h * j0), (h * (i0 + sx), h * (j0 + sy)),
                        (h * i0, h * (j0 + sy))])
        x0 = d.initial_state()
        n = p.n_interior
        noise = 0.01 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
        x0.psi[:] += noise * (d.material.interior_sc_mask if d.material is not None else 1.0)
        devs.append(d)
        xs.append(x0.data.copy())
        desc.append((Nx, Ny, Nz, nh))
    return devs, xs, desc


def batched_shard(sizes, rank: int, world: int) -> list:
    """Instances of this rank: the 64 split over the ranks largest first,
    each to the rank with the fewest interior nodes so far (independent
    instances: no data moves between ranks)."""
    from nanowire_tdgl_b200.batch import assign_streams
    return sorted(assign_streams(sizes, world)[0][rank])


def run_batched(a, rank: int = 0, world: int = 1):
    """Instance-steps/s of the 64 instances stepped together (autotuned launch
    shapes, one stream per instance) against looping them one after another with the
    single-instance launch shapes; both device-timed over the same K steps per
    instance after W warm-up steps, from the same states.  Under torchrun the
    instances are split over the ranks and the job time is the slowest
    rank's."""
    import torch
    import nanowire_tdgl_b200 as tb
    devs, xs, desc = batched_workload()
    n_all = len(devs)
    node_total = sum(d.params.n_interior for d in devs)
    if world > 1:
        mine = batched_shard([d.params.n_interior for d in devs], rank, world)
        devs, xs, desc = [devs[i] for i in mine], [xs[i] for i in mine], [desc[i] for i in mine]
    dist = world > 1
    n_nodes = [d.params.n_interior for d in devs]
    kw = dict(precision="mixed", kmax=a.kmax, newton_tol_f=1e-8, newton_tol_dx=1e-3, tol_gcr=1e-6, eps_mf=1e-4)
    bt = tb.BatchedTrapezoidal(devs, xs, BATCH["dt"], n_streams=64, **kw)
    clocks = Clocks()
    clocks.start()
    tune = bt.autotune(steps=2)
    bt.step(a.warmup)
    tot0 = dict(bt.totals)
    if dist:
        torch.distributed.barrier()
    ms_b = max_over_ranks(bt.time_steps(a.steps), dist, "cuda")
    cnt = {k: bt.totals[k] - tot0[k] for k in tot0}
    states_b = bt.states()
    # looping baseline: the single-instance launch shapes, one instance after another
    lp = tb.BatchedTrapezoidal(devs, xs, BATCH["dt"], **kw)
    lp.set_shape(None)
    lp.step_sequential(a.warmup)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    lp.step_sequential(a.steps)
    e1.record()
    torch.cuda.synchronize()
    ms_l = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(0).uuid)
    except Exception:
        pass
    clk = clocks.stop(uuid)
    rel = []
    for d, u, v in zip(devs, states_b, lp.states()):
        n = d.params.n_interior
        pu, pv = np.abs(u[:n]) ** 2, np.abs(v[:n]) ** 2
        rel.append(float(np.linalg.norm(pu - pv) / np.linalg.norm(pv)))
    free, total = torch.cuda.mem_get_info()
    inst_steps = n_all * a.steps
    return {"form": "batched", "metric": "instance-steps/s, 64 seeded uneven instances, batched vs looping",
            "value": inst_steps / (ms_b / 1e3), "unit": "instance-steps/s",
            "looping_value": inst_steps / (ms_l / 1e3), "speedup_vs_looping": ms_l / ms_b,
            "steps_per_instance": a.steps, "warmup": a.warmup, "ms_batched": ms_b, "ms_looping": ms_l,
            "node_updates_per_s": node_total * a.steps / (ms_b / 1e3), "n_gpus": world,
            "scaling": "strong" if dist else "single GPU",
            "dtype": "f32 Krylov / f64 state", "data": "synthetic (seeded instances)",
            "config": {"workload": "64 instances, Nx,Ny in {32,48,64,96}, Nz in {4,8,16}, h 0.5, kappa U[1.5,4], "
                                   "Bz U[0.1,1], 0-3 rectangular holes of side 4-16 nodes, dt 0.1, Newton tol_f "
                                   "1e-8 / tol_dx 1e-3, GMRES tol 1e-6",
                       "interior_nodes_total": sum(n_nodes), "interior_nodes_min": min(n_nodes),
                       "interior_nodes_max": max(n_nodes), "holes_total": sum(q[3] for q in desc),
                       "streams": len(bt.streams), "kmax": a.kmax},
            "autotune_ms_per_2_steps": {f"{k[0]} nodes/thread, {'one' if k[1] else 'two'} kernel(s)"
                                        + (f", degree {k[2]}" if len(k) > 2 else ""): v
                                        for k, v in tune.items()},
            "shape": {"nodes_per_thread": bt.best[0], "fused_product_projections": bool(bt.best[1]),
                      "poly_degree": bt.best[2] if len(bt.best) > 2 else None},
            "counters": cnt,
            "max_rel_l2_psi2_batched_vs_looping": max_over_ranks(max(rel), dist, "cuda"),
            "note": "batched and looping differ in launch shapes (reduction partitions) and, when the autotuner "
                    "picks another degree than the single-instance default 10, in the preconditioner (converged states agree to "
                    "the Newton tolerance); at equal shapes and degree the results are bit-identical",
            "device_memory_in_use_gb": (total - free) / 1e9,
            "clocks": clk}


TRI = dict(Nx=256, Ny=256, layers=(24, 16, 24), h=0.5, kappa=4.0, Bz=0.6,
           hole=[(48, 48), (80, 48), (80, 80), (48, 80)], dt=0.1, seed=13, t_stop=200.0, kmax=160)


def trilayer_device():
    """256x256x64-cell superconductor / insulator / superconductor stack (24 /
    16 / 24 cells in z, kappa 4 everywhere, psi relaxed in the insulator),
    centred 64x64-node hole through all layers, Bz 0.6, seeded psi0 noise
    0.01 on the superconducting nodes, phi0 = 0."""
    import nanowire_tdgl_b200 as tb
    w = TRI
    b, i, t = w["layers"]
    p = tb.SimulationParameters(Nx=w["Nx"], Ny=w["Ny"], Nz=b + i + t, hx=w["h"], hy=w["h"], hz=w["h"],
                                kappa=w["kappa"])
    tri = tb.Trilayer(tb.Layer(b, w["kappa"]), tb.Layer(i, w["kappa"], is_superconductor=False),
                      tb.Layer(t, w["kappa"]))
    dev = tb.Device(p, applied_field=tb.AppliedField(Bz=w["Bz"], t_on_fraction=1.0), trilayer=tri)
    dev.add_hole(w["hole"])
    rng = np.random.default_rng(w["seed"])
    x0 = dev.initial_state()
    n = p.n_interior
    x0.psi[:] += 0.01 * (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * dev.material.interior_sc_mask
    return dev, x0.data.copy()


def run_trilayer(a):
    """Steps/s, roofline fraction and error against the FP64 stepper (the
    reference's finite-difference product) of the mixed stepper on the large
    trilayer, over the same K steps after W warm-up steps."""
    import torch
    from nanowire_tdgl_b200 import _lib as L
    from nanowire_tdgl_b200.engine import grid_for
    w = TRI
    dev, x0 = trilayer_device()
    p = dev.params
    n_int = p.n_interior
    runs = {}
    for prec, jvp in (("mixed", L.TDGL_JVP_ANALYTIC), ("fp64", L.TDGL_JVP_FD)):
        g = grid_for(p, dev.idx, dev.material, prec, w["kmax"], "gmres")
        opts = L.TrapOpts(w["t_stop"], w["dt"], 1e-8, 1e-8, 1e-3, 1e-6, 1e-4, 20, 0, 1, jvp)
        fld = L.Field(0.0, 0.0, w["Bz"], 1.0, 0.5, w["t_stop"], 0, 0)
        x, ms, st = device_run(g, x0, opts, fld, a.warmup, a.steps, False)
        runs[prec] = (g, x, ms, st)
    (gm, xm, msm, stm), (gd, xd, msd, std) = runs["mixed"], runs["fp64"]
    B = (0.0, 0.0, w["Bz"])
    om, od = gm.observables(xm, B), gd.observables(xd, B)
    def rel(k):
        return float(torch.linalg.vector_norm(om[k] - od[k]) / torch.linalg.vector_norm(od[k]))
    peak, peak_kind = measured_peak()
    alg = algorithmic_bytes(n_int, "mixed", stm, gm.poly_degree)
    achieved = alg / (msm / 1e3) / 1e9
    return {"form": "trilayer", "metric": "trapezoidal steps/s, 256x256x64 S/I/S trilayer, mixed vs FP64",
            "value": a.steps / (msm / 1e3), "unit": "steps/s", "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": msm / a.steps, "node_updates_per_s": n_int * a.steps / (msm / 1e3),
            "fp64_value": a.steps / (msd / 1e3), "speedup_vs_fp64": msd / msm,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": None, "algorithmic_bytes_per_launch": alg,
                         "traffic_note": "not captured at this size (the film's ratio does not carry over: its preconditioned basis stays in L2, this one does not)"},
            "rel_l2_vs_fp64": {"psi2": rel("psi2"), "Bz": rel("Bz"), "Jx": rel("Jx"), "Jy": rel("Jy")},
            "max_abs_psi2_vs_fp64": float((om["psi2"] - od["psi2"]).abs().max()),
            "dtype": "f32 Krylov / f64 state", "data": "synthetic (seeded psi0 noise)",
            "config": {"workload": "256x256x64 cells, S/I/S 24/16/24 in z, kappa 4, Bz 0.6, centred 64x64-node "
                                   "hole through all layers, dt 0.1, Newton tol_f 1e-8 / tol_dx 1e-3, GMRES tol "
                                   "1e-6, kmax 160", "n_interior": n_int},
            "counters": {k: stm[k] for k in ("newton_iters", "krylov_iters", "rejections", "max_krylov")},
            "fp64_counters": {k: std[k] for k in ("newton_iters", "krylov_iters", "rejections", "max_krylov")}}


def run_forms(a) -> dict:
    """The other forms of the build, measured after the headline line of the
    default run (one GPU), each at a reduced step count and guarded so that a
    failure leaves the headline intact: the 256x256x64 trilayer (3 steps after
    1 warm-up), the 64-instance batch (4 steps per instance after 1 warm-up,
    autotuned), and the differentiation workload (400 steps forward and
    adjoint) at s(x) in [0, 0.05] and at the configured [0, 1]."""
    import gc
    import torch
    from nanowire_tdgl_b200 import engine
    res = {}
    def fresh():
        engine._CACHE.clear()
        gc.collect()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    def sub(**kw):
        b = argparse.Namespace(**vars(a))
        for k, v in kw.items():
            setattr(b, k, v)
        return b
    jobs = [("trilayer", lambda: run_trilayer(sub(steps=3, warmup=1))),
            ("batched", lambda: run_batched(sub(steps=4, warmup=1))),
            ("adjoint", lambda: run_adjoint(a, 0.05)),
            ("adjoint_s_0_to_1", lambda: run_adjoint(a, 1.0))]
    for name, job in jobs:
        fresh()
        t0 = time.perf_counter()
        try:
            r = job()
        except Exception as e:                        # keep the headline line whatever a form does
            r = {"error": f"{type(e).__name__}: {e}"}
        r["wall_s"] = time.perf_counter() - t0
        res[name] = r
    fresh()
    deg = res.get("adjoint_s_0_to_1", {})
    if "loss" in deg:
        deg["note"] = ("with s(x) up to 1 the reference's relaxation -(1 - sc) psi / 0.1 (sc = 1 - s) drives psi "
                       "to ~0 wherever s exceeds ~0.1, so the box loss is ~0 and its finite differences are "
                       "round-off; the gradient check is the [0, 0.05] run")
    return res


def main():
    a = parse()
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")   # before CUDA starts: one queue per batch stream
    if a.form == "trilayer":
        print(json.dumps(run_trilayer(a)), flush=True)
        return 0
    if a.form == "adjoint":
        print(json.dumps(run_adjoint(a, a.adj_smax)), flush=True)
        return 0
    if a.form == "batched":
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")   # before CUDA is initialised
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        if world > 1:
            import torch
            from datetime import timedelta
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
            torch.distributed.init_process_group("nccl", timeout=timedelta(seconds=300))
        try:
            out = run_batched(a, rank, world)
        finally:
            if world > 1:
                torch.distributed.destroy_process_group()
        if rank == 0:
            print(json.dumps(out), flush=True)
        return 0
    if a.arnoldi_probe is not None:
        return arnoldi_probe(a)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if a.impl == "reference":
        out = run_reference(a, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return 0
    import torch
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=timedelta(seconds=300))
    try:
        out = run_ours(a, rank, world)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()
    x1 = out.pop("_x1", None)
    if rank == 0:
        if world == 1 and not a.no_cpu_baseline:
            done, el, xo = cpu_oracle_steps(1, a.cpu_budget_s, 1, want_state=True)
            out["cpu_baseline"] = {"value": done / el, "unit": "steps/s", "cores": 1, "kind": "port",
                                   "sample": f"{done} trapezoidal step(s) from the seeded state (step 1), numpy "
                                             "oracle restating the reference algorithm, 1 thread"}
            if x1 is not None and xo is not None:
                n = WORKLOAD_N_INTERIOR
                p2, p2o = np.abs(x1[:n]) ** 2, np.abs(xo[:n]) ** 2
                out["rel_l2_psi2_vs_oracle"] = float(np.linalg.norm(p2 - p2o) / np.linalg.norm(p2o))
                out["max_abs_vs_oracle"] = float(np.max(np.abs(x1 - xo)))
                out["vs_oracle_note"] = (f"state after step 1 from the seeded state: this run's {a.precision} "
                                         "stepper against the oracle's FP64 finite-difference GCR step (same "
                                         "tolerances); max_abs over all state entries")
        if world == 1 and not a.no_forms:
            out["forms"] = run_forms(a)
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
