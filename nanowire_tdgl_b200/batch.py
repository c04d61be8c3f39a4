"""Batched form: many independent instances stepped together on one GPU.

Each instance (its own grid size, field, holes, kappa) keeps its own device
context and trapezoidal step graph (the whole step loop, Newton and GMRES
iterations under conditional graph nodes).  ``BatchedTrapezoidal.step``
enqueues every instance's graph on one of a set of CUDA streams and only then
waits, so the GPU runs the instances' kernels concurrently: small instances,
which leave most SMs idle when stepped one at a time, fill the machine
together.  Instances are assigned to streams largest first, each to the
stream with the least work so far.

The autotuner chooses the launch shape of every instance's grid kernels: a
candidate is a number of nodes per thread, from which each instance's block
count follows from its size (the single-instance default of 8 blocks per SM
for the grid-stride passes and 5 for the Arnoldi streams is one candidate),
and whether each Arnoldi iteration runs the product and the projections as
one kernel or two (fewer, longer launches help small instances, whose
kernels are launch-bound).  Each candidate is timed over a few batched steps
from a snapshot of the states, which is restored afterwards.

Each instance's arithmetic is its single-instance arithmetic (the same
kernels, fixed-order reductions), so the results equal those of stepping the
instances one after another with the same launch shapes, bit for bit.

More than 8 streams only run concurrently when ``CUDA_DEVICE_MAX_CONNECTIONS``
(default 8) is raised before CUDA is initialised; ``bench.py`` sets it to 32.
"""

from __future__ import annotations

import math
from typing import Optional, Sequence

import torch

from . import _lib as L
from .engine import DeviceGrid

_THREADS = 256                  # threads per block of the step graph's kernels


def assign_streams(sizes: Sequence[int], n_streams: int) -> tuple[list, list]:
    """Instances (by size) to streams, largest first, each to the stream with
    the least work so far.  Returns (queues, order): the instance indices of
    each stream, and the launch order (stream, instance) that takes the first
    instance of every stream, then the second, ..."""
    ns = max(1, min(int(n_streams), len(sizes)))
    load = [0] * ns
    queues = [[] for _ in range(ns)]
    for i in sorted(range(len(sizes)), key=lambda i: -sizes[i]):
        s = min(range(ns), key=load.__getitem__)
        queues[s].append(i)
        load[s] += sizes[i]
    depth = max(len(q) for q in queues)
    order = [(s, q[r]) for r in range(depth) for s, q in enumerate(queues) if r < len(q)]
    return queues, order


def instance_field(applied_field, t_stop: float, schedule: bool) -> L.Field:
    """Device field of one instance.  Without ``schedule``: the constant
    (Bx, By, Bz) of its ``AppliedField`` at every step.  With it: the
    ``AppliedField`` schedule against ``t_stop`` (zero at t <= 0 and after
    t_stop * t_on_fraction, the optional ramp), evaluated at each step's
    start as the reference's step loop does (src/tdgl3d/solvers/
    integrators.py:150-153, physics/applied_field.py:42-56); a Python
    ``field_func`` cannot be evaluated on the device (ValueError)."""
    af = applied_field
    if not schedule:
        return L.Field(float(af.Bx), float(af.By), float(af.Bz), 1.0, 0.0, float(t_stop), 0, 1)
    if getattr(af, "field_func", None) is not None:
        raise ValueError("field_schedule needs an AppliedField without field_func")
    if not math.isfinite(t_stop):
        raise ValueError("field_schedule needs a finite t_stop")
    return L.Field(float(af.Bx), float(af.By), float(af.Bz), float(af.t_on_fraction), float(af.ramp_fraction),
                   float(t_stop), int(bool(af.ramp)), 0)


def launch_blocks(n: int, nodes_per_thread: Optional[int], sms: int) -> tuple[int, int]:
    """(grid-stride blocks, Arnoldi blocks) of an instance of n interior
    nodes: the single-instance default (8 and 5 blocks per SM) for None, else
    enough blocks for ``nodes_per_thread`` nodes a thread, capped there."""
    if nodes_per_thread is None:
        return 8 * sms, 5 * sms
    b = max(1, min(8 * sms, math.ceil(n / (_THREADS * nodes_per_thread))))
    return b, max(1, min(5 * sms, math.ceil(b * 5 / 8)))


class BatchedTrapezoidal:
    """Trapezoidal stepping of ``devices`` (``Device`` objects, distinct) from
    the reference-layout states ``x0s``, each with its device's constant
    applied field (Bx, By, Bz of its ``AppliedField``), or, with
    ``field_schedule``, with its ``AppliedField`` schedule against
    ``t_stop`` as ``solve`` applies it (``instance_field``)."""

    def __init__(self, devices: Sequence, x0s: Sequence, dt: float, *, t_start: float = 0.0,
                 t_stop: float = 1e30, precision: str = "mixed", kmax: int = 64, newton_tol_f: float = 1e-8,
                 newton_tol_dx: float = 1e-3, newton_max_iter: int = 20, tol_gcr: float = 1e-6,
                 eps_mf: float = 1e-4, adaptive: bool = True, dt_min: float = 1e-8, n_streams: int = 32,
                 field_schedule: bool = False):
        if len({id(d) for d in devices}) != len(devices):
            raise ValueError("every instance needs its own Device object")
        fields = [instance_field(d.applied_field, t_stop, field_schedule) for d in devices]
        # contexts of their own (not the per-device cache): their launch shapes are the batch's
        self.grids = [DeviceGrid(d.params, d.idx, d.material, precision, kmax, "gmres") for d in devices]
        self.x = [g.pack(x0) for g, x0 in zip(self.grids, x0s)]
        torch.cuda.synchronize()
        self.t = [float(t_start)] * len(devices)
        self.cur = [float(dt)] * len(devices)
        jvp = L.TDGL_JVP_ANALYTIC if precision == "mixed" else L.TDGL_JVP_FD
        self.opts = L.TrapOpts(float(t_stop), float(dt), float(dt_min), float(newton_tol_f), float(newton_tol_dx),
                               float(tol_gcr), float(eps_mf), int(newton_max_iter), 0, int(bool(adaptive)), jvp)
        self.fields = fields
        self.totals = {"steps": 0, "newton_iters": 0, "krylov_iters": 0, "rejections": 0}
        self.sms = torch.cuda.get_device_properties(self.grids[0].device).multi_processor_count
        self.shape = (None, -1)                # (nodes per thread or None: single-instance shapes, fused)
        self.best = None                       # the autotuner's choice
        self.set_streams(n_streams)

    def __len__(self) -> int:
        return len(self.grids)

    # -- scheduling -----------------------------------------------------------
    def set_streams(self, n_streams: int) -> None:
        """Spread the instances over ``n_streams`` streams (``assign_streams``)."""
        self.queues, self.order = assign_streams([g.n for g in self.grids], n_streams)
        self.streams = [torch.cuda.Stream(device=self.grids[0].device) for _ in self.queues]

    def set_shape(self, nodes_per_thread: Optional[int], fused: int = -1, poly: Optional[int] = None) -> None:
        """Launch shape of every instance: blocks from ``nodes_per_thread``
        (``launch_blocks``); Arnoldi product and projections as one kernel
        (fused 1), two (0) or the precision's default (-1); and, when given,
        the degree of the polynomial preconditioner (-1: the default; None
        leaves it as it is)."""
        for g in self.grids:
            g.set_blocks(*launch_blocks(g.n, nodes_per_thread, self.sms), fused)
            if poly is not None:
                g.set_poly(poly)
        self.shape = (nodes_per_thread, fused) if poly is None else (nodes_per_thread, fused, poly)

    # -- stepping ---------------------------------------------------------------
    def _account(self, rc: int, t: float, cur: float, st: dict, i: int) -> None:
        L.check(rc, f"instance {i}")
        self.t[i], self.cur[i] = t, cur
        for k in self.totals:
            self.totals[k] += st[k]

    def step(self, n_steps: int) -> None:
        """n_steps accepted steps of every instance, all streams in flight
        together.  The streams start after the work already queued on the
        current stream and the current stream waits for all of them, so CUDA
        events recorded on it around this call time the batch."""
        cur = torch.cuda.current_stream(self.grids[0].device)
        for s in self.streams:
            s.wait_stream(cur)
        launched = []
        try:
            for s, i in self.order:
                self.grids[i].trap_launch(self.x[i], self.t[i], self.cur[i], n_steps, self.opts, self.fields[i],
                                          self.streams[s])
                launched.append(i)
        finally:                               # every launched context is collected, even after an error
            for s in self.streams:
                cur.wait_stream(s)
            for s in self.streams:
                s.synchronize()
            results = [(i, self.grids[i].trap_collect()) for i in launched]
        for i, r in sorted(results, key=lambda e: e[0]):
            self._account(*r, i)

    def step_sequential(self, n_steps: int) -> None:
        """The same steps one instance after another on the current stream,
        each waited for (the looping baseline)."""
        for i, g in enumerate(self.grids):
            self._account(*g.trap_run(self.x[i], self.t[i], self.cur[i], n_steps, self.opts, self.fields[i]), i)

    # -- autotuning -------------------------------------------------------------
    def snapshot(self):
        torch.cuda.synchronize()
        return [x.clone() for x in self.x], list(self.t), list(self.cur), dict(self.totals)

    def restore(self, snap) -> None:
        xs, ts, curs, tot = snap
        for x, y in zip(self.x, xs):
            x.copy_(y)
        torch.cuda.synchronize()
        self.t, self.cur, self.totals = list(ts), list(curs), dict(tot)

    def time_steps(self, n_steps: int) -> float:
        """Device time (ms) of ``n_steps`` batched steps."""
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        self.step(n_steps)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def autotune(self, candidates: Sequence = tuple((n, f, p) for n in (None, 1, 2, 4, 8) for f in (0, 1)
                                                    for p in (5, 8, 10)),
                 steps: int = 2) -> dict:
        """Time ``steps`` batched steps from the current states for each
        (nodes per thread, fused[, preconditioner degree]) candidate
        (``set_shape``), after one untimed step that builds the graphs; keep
        the fastest.  States, clocks and counters are restored.  Returns
        {candidate: ms}.  (Stiffer instances, larger kappa^2 dt / h^2, gain
        from the higher degree: on the 64-instance workload degree 5 stepped
        9 % faster than degree 3 and degree 8 ~3 % faster than 5 at the
        chosen shape; 10 is the single-instance default.)"""
        snap = self.snapshot()
        times = {}
        for cand in candidates:
            self.set_shape(*cand)
            self.step(1)
            self.restore(snap)
            times[cand] = self.time_steps(steps)
            self.restore(snap)
        self.best = min(times, key=times.get)
        self.set_shape(*self.best)
        return times

    def states(self) -> list:
        """Reference-layout complex128 states (numpy)."""
        return [g.unpack(x).cpu().numpy() for g, x in zip(self.grids, self.x)]
