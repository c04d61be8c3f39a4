"""Drop-in solver entry points with the signatures of tdgl3d's hot path.

==========================  ===============================================
this module                 reference (paths inside the tdgl3d project)
==========================  ===============================================
``eval_f``                  src/tdgl3d/physics/rhs.py:147-239
``make_eval_f``             src/tdgl3d/solvers/integrators.py:23-32
``tgcr_matrix_free_trap``   src/tdgl3d/solvers/tgcr.py:96-156
``newton_gcr_trap``         src/tdgl3d/solvers/newton.py:76-120
``trapezoidal``             src/tdgl3d/solvers/integrators.py:92-206
``forward_euler``           src/tdgl3d/solvers/integrators.py:35-89
``solve``                   src/tdgl3d/solvers/runner.py:40-163
==========================  ===============================================

Arrays in and out are reference-layout complex128 state vectors (numpy on
the host, or torch tensors, which are returned as torch tensors on the
device).  The numerics run in the CUDA kernels of ``libtdgl_b200.so``.

``tgcr_matrix_free_trap`` and ``newton_gcr_trap`` keep the reference's
generic contract: given this package's device RHS (``make_eval_f``) the whole
solve runs on the device; given any other Python callable they run the
reference algorithm with the vectors on the GPU (torch) and call the
callable for every function value.

Keyword-only additions: ``precision`` ("fp64" | "mixed"), ``jvp`` ("fd" |
"analytic"), ``krylov`` ("gmres" | "gcr": the same minimal-residual iterates,
GMRES storing one vector per iteration instead of GCR's two) and ``kmax``
(Krylov directions held on the device).  The default Krylov method follows
the product: with the reference's finite-difference product (the FP64
default) it is the reference's own GCR (src/tdgl3d/solvers/tgcr.py:96-156),
so a script switched over to this package gets the reference's method
unless it asks for another; with analytic products (the mixed-precision
default) it is GMRES with the polynomial preconditioner, the fast path.
"""

from __future__ import annotations

import ctypes
import json
import mmap
import os
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from datetime import datetime
from pathlib import Path
from typing import Callable, Optional

import numpy as np
import torch

from . import _lib as L
from .engine import grid_for
from .model import (AppliedField, BoundaryVectors, StateVector, build_boundary_field_vectors,
                    field_scalars_from_vectors)

DEFAULT_KMAX = 64


def default_krylov(krylov: Optional[str], jvp: str) -> str:
    """The Krylov method of a call: as given, else GCR (the reference's) for
    finite-difference products and GMRES for analytic ones."""
    if krylov is not None:
        return krylov
    return "gcr" if jvp == "fd" else "gmres"


def _is_torch(x) -> bool:
    return isinstance(x, torch.Tensor)


def _out(t: torch.Tensor, like):
    if _is_torch(like):
        return t
    return t.cpu().numpy()


class DeviceRHS:
    """f(X) = dX/dt for fixed (params, idx, material, applied field) — the
    closure ``_make_eval_f`` returns in the reference, evaluated on the GPU.
    Passing it to :func:`tgcr_matrix_free_trap` / :func:`newton_gcr_trap`
    keeps the whole solve on the device."""

    def __init__(self, params, idx, B, material=None, precision: str = "fp64", jvp: Optional[str] = None,
                 kmax: int = DEFAULT_KMAX, krylov: Optional[str] = None):
        self.params, self.idx, self.material = params, idx, material
        self.B = tuple(float(b) for b in B)
        self.precision = precision
        self.jvp = jvp or ("fd" if precision == "fp64" else "analytic")
        self.grid = grid_for(params, idx, material, precision, kmax, default_krylov(krylov, self.jvp))

    def __call__(self, X):
        return _out(self.grid.eval_f_ref(X, self.B), X)


def make_eval_f(params, idx, u, material=None, **kw) -> DeviceRHS:
    """Device counterpart of ``_make_eval_f`` (integrators.py:23-32)."""
    B = field_scalars_from_vectors(u, params, idx) if isinstance(u, BoundaryVectors) or hasattr(u, "Bz") else u
    return DeviceRHS(params, idx, B, material, **kw)


def eval_f(X, params, idx, u, material=None):
    """dX/dt of the state X (rhs.py:147-239).  ``u`` is the reference's
    BoundaryVectors (applied field on the boundary faces) or a (Bx, By, Bz)
    tuple."""
    B = field_scalars_from_vectors(u, params, idx) if hasattr(u, "Bz") else tuple(u)
    g = grid_for(params, idx, material, "fp64", DEFAULT_KMAX)
    _check_real_links(X, params)
    return _out(g.eval_f_ref(X, B), X)


def _check_real_links(X, params) -> None:
    n = params.n_interior
    if _is_torch(X):
        if X.is_complex() and bool(torch.any(X[n:].imag != 0)):
            raise ValueError("link variables must be real (imaginary part of phi is nonzero)")
    else:
        a = np.asarray(X)
        if np.iscomplexobj(a) and np.any(a[n:].imag != 0):
            raise ValueError("link variables must be real (imaginary part of phi is nonzero)")


# ---------------------------------------------------------------------------
# Krylov and Newton
# ---------------------------------------------------------------------------

def tgcr_matrix_free_trap(eval_f: Callable, x_lin, b, dt: float, tol: float = 1e-4,
                          max_iter: Optional[int] = None, eps_mf: float = 1e-4):
    """Solve (I - dt/2 J(x_lin)) d = b (tgcr.py:96-156); returns d, or an
    empty array when the relative residual stays above ``tol``."""
    if isinstance(eval_f, DeviceRHS):
        g = eval_f.grid
        x = g.pack(x_lin)
        bd = g.pack(b)
        if max_iter is not None and int(max_iter) <= 0:
            # no iteration allowed: the reference returns zeros when b == 0 or
            # tol >= 1, and fails otherwise
            bn = float(torch.linalg.vector_norm(g.ref_tensor(b)))
            if bn == 0.0 or not (bn > tol * bn):
                return _out(torch.zeros(g.n_state, dtype=torch.complex128, device=g.device), b)
            return _empty_like(b)
        mi = 0 if max_iter is None else int(max_iter)   # 0: the reference default len(b)
        d, st = g.tgcr(x, bd, dt, tol, mi, eps_mf, eval_f.jvp, eval_f.B)
        if d is None:
            return _empty_like(b)
        return _out(g.unpack(d), b)
    return _generic_tgcr_trap(eval_f, x_lin, b, dt, tol, max_iter, eps_mf)


def newton_gcr_trap(eval_f: Callable, x0, gamma, dt: float, *, tol_f: float = 1e-3, tol_dx: float = 1e-3,
                    max_iter: int = 20, tol_gcr: float = 1e-4, eps_mf: float = 1e-4, verbose: bool = False):
    """Newton on g(x) = x - dt/2 f(x) - gamma (newton.py:76-120); returns
    (x, converged, iterations)."""
    if isinstance(eval_f, DeviceRHS):
        g = eval_f.grid
        x = g.pack(x0)
        gm = g.pack(gamma)
        st = g.newton(x, gm, dt, tol_f, tol_dx, max_iter, tol_gcr, eps_mf, eval_f.jvp, eval_f.B)
        if verbose:
            print(f"  Newton-Trap: ||g||inf = {st['last_gnorm']:.3e}, ||dx||inf = {st['last_dxnorm']:.3e}")
        return _out(g.unpack(x), x0), bool(st["newton_converged"]), int(st["newton_iters_last"])
    return _generic_newton_trap(eval_f, x0, gamma, dt, tol_f, tol_dx, max_iter, tol_gcr, eps_mf, verbose)


def _empty_like(like):
    if _is_torch(like):
        return torch.empty(0, dtype=torch.complex128, device=like.device)
    return np.array([], dtype=np.complex128)


def _gpu(x) -> torch.Tensor:
    if not torch.cuda.is_available():
        raise RuntimeError("nanowire_tdgl_b200 needs a CUDA device")
    if _is_torch(x):
        return x.to("cuda", torch.complex128)
    return torch.from_numpy(np.asarray(x, dtype=np.complex128).copy()).to("cuda")


def _call(f, x: torch.Tensor, like) -> torch.Tensor:
    arg = x if _is_torch(like) else x.cpu().numpy()
    return _gpu(f(arg))


def _generic_tgcr_trap(f, x_lin, b, dt, tol, max_iter, eps_mf):
    """The reference TGCR for an arbitrary Python RHS, vectors on the GPU."""
    bb = _gpu(b)
    xl = _gpu(x_lin)
    N = bb.numel()
    if max_iter is None:
        max_iter = max(N, int(round(0.2 * N)))
    x = torch.zeros_like(bb)
    r = bb.clone()
    r0 = float(torch.linalg.vector_norm(r))
    rn = r0
    if r0 == 0.0:
        return _out(x, b)
    P, AP = [], []
    f_base = _call(f, xl, b)
    xn = float(torch.linalg.vector_norm(xl))
    k = 0
    while rn / r0 > tol and k < max_iter:
        k += 1
        p = r.clone()
        eps = eps_mf * (1.0 + xn) / float(torch.linalg.vector_norm(p))
        ap = p - (dt / 2.0) * ((_call(f, xl + eps * p, b) - f_base) / eps)
        for pj, apj in zip(P, AP):
            beta = float(torch.vdot(ap, apj).real)
            p = p - beta * pj
            ap = ap - beta * apj
        nap = float(torch.linalg.vector_norm(ap))
        if nap < 1e-14:
            break
        ap = ap / nap
        p = p / nap
        P.append(p)
        AP.append(ap)
        alpha = float(torch.vdot(r, ap).real)
        x = x + alpha * p
        r = r - alpha * ap
        rn = float(torch.linalg.vector_norm(r))
    if rn > tol * r0:
        return _empty_like(b)
    return _out(x, b)


def _generic_newton_trap(f, x0, gamma, dt, tol_f, tol_dx, max_iter, tol_gcr, eps_mf, verbose):
    x = _gpu(x0)
    gm = _gpu(gamma)
    for k in range(1, max_iter + 1):
        g = x - (dt / 2.0) * _call(f, x, x0) - gm
        dx = _generic_tgcr_trap(f, x if _is_torch(x0) else x.cpu().numpy(), -g if _is_torch(x0) else (-g).cpu().numpy(),
                                dt, tol_gcr, None, eps_mf)
        if len(dx) == 0:
            if verbose:
                print(f"  Newton-Trap iter {k}: GCR did not converge")
            return _out(x, x0), False, k
        x = x + _gpu(dx)
        g = x - (dt / 2.0) * _call(f, x, x0) - gm
        errf = float(torch.max(torch.abs(g))) if g.numel() else 0.0
        err_dx = float(torch.max(torch.abs(_gpu(dx)))) if len(dx) else 0.0
        if verbose:
            print(f"  Newton-Trap iter {k}: ||g||inf = {errf:.3e}, ||dx||inf = {err_dx:.3e}")
        if errf <= tol_f and err_dx <= tol_dx:
            return _out(x, x0), True, k
    return _out(x, x0), False, max_iter


# ---------------------------------------------------------------------------
# Time stepping
# ---------------------------------------------------------------------------

class FieldSchedule:
    """``eval_u(t, X)`` of an AppliedField (runner.py:24-37) that the device
    can evaluate itself; calling it returns reference BoundaryVectors."""

    def __init__(self, applied_field: AppliedField, params, idx, t_stop: float):
        self.applied_field, self.params, self.idx, self.t_stop = applied_field, params, idx, float(t_stop)

    def __call__(self, t, X=None):
        bx, by, bz = self.applied_field.evaluate(t, self.t_stop)
        return BoundaryVectors(*build_boundary_field_vectors(bx, by, bz, self.params, self.idx))

    def device_field(self) -> Optional[L.Field]:
        af = self.applied_field
        if getattr(af, "field_func", None) is not None:
            return None
        return L.Field(float(af.Bx), float(af.By), float(af.Bz), float(af.t_on_fraction),
                       float(af.ramp_fraction), self.t_stop, int(bool(af.ramp)), 0)


def _count_steps(t_start: float, t_stop: float, dt: float) -> int:
    """Steps of min(dt, t_stop - t) while t < t_stop - 1e-14 (no retries)."""
    t, n = float(t_start), 0
    while t < t_stop - 1e-14 and n < 100_000_000:
        t += min(dt, t_stop - t)
        n += 1
    return n


def _host_rows(rows: int, n: int) -> torch.Tensor:
    """(rows, n) complex128 host tensor for the saved states.  Large outputs
    are placed on an anonymous mapping advised for transparent huge pages: the
    first write into each page pays a fault, and with 2 MB pages the landing
    copies run at about 1.5x the rate they reach with 4 KB pages (measured
    20 against 13 GB/s on 8 threads).  Falls back to an ordinary allocation."""
    nbytes = rows * n * 16
    if nbytes >= (16 << 20) and hasattr(mmap, "MADV_HUGEPAGE"):
        try:
            buf = mmap.mmap(-1, nbytes, flags=mmap.MAP_PRIVATE | mmap.MAP_ANONYMOUS)
            buf.madvise(mmap.MADV_HUGEPAGE)
            arr = np.frombuffer(buf, dtype=np.complex128).reshape(rows, n)
            return torch.from_numpy(arr)
        except (OSError, ValueError):
            pass
    return torch.empty((rows, n), dtype=torch.complex128)


class _History:
    """Saved states on their way to host memory while the device steps on.

    stage(x): the state is unpacked into one of NBUF device staging buffers on
    the compute stream (in stream order, before a later launch changes x) and
    copied asynchronously on a side stream into pinned host staging; the
    token it returns is then either committed as row k of the output (a
    worker thread copies it there once the copy has landed) or discarded.
    save(x) stages and commits at once.  The output is preallocated for the
    expected number of saves; rows beyond it, after dt retries, are appended.
    The host copy runs as several memmove calls on a small thread pool: they
    release the GIL (a torch CPU copy holds it, stalling the stepping thread
    for its whole duration) and share the page faults of the fresh output
    rows.  The host-side copies overlap the next device launches.
    """

    COPY_THREADS = max(1, min(8, (os.cpu_count() or 1) // 2))
    NBUF = 3

    def __init__(self, g, rows: int):
        self.g = g
        self.rows = _host_rows(max(rows, 1), g.n_state)
        self.extra: list[torch.Tensor] = []
        self.n = 0
        self.nstaged = 0
        st = getattr(g, "_history_staging", None)
        if st is None or len(st["dev"]) < self.NBUF:
            st = {"dev": [torch.empty(g.n_state, dtype=torch.complex128, device=g.device) for _ in range(self.NBUF)],
                  "pin": [torch.empty(g.n_state, dtype=torch.complex128, pin_memory=True)
                          for _ in range(self.NBUF)],
                  "stream": torch.cuda.Stream(device=g.device)}
            g._history_staging = st
        self.st = st
        self.ready = [torch.cuda.Event() for _ in range(self.NBUF)]
        self.copied = [torch.cuda.Event() for _ in range(self.NBUF)]
        self.futs = [None] * self.NBUF
        self.pool = ThreadPoolExecutor(max_workers=1)
        self.copy_pool = ThreadPoolExecutor(max_workers=self.COPY_THREADS)
        self.lock = threading.Lock()

    def stage(self, x: torch.Tensor) -> int:
        k = self.nstaged % self.NBUF
        self.nstaged += 1
        if self.futs[k] is not None:
            self.futs[k].result()
            self.futs[k] = None
        st = self.st
        # the side-stream copy of this buffer's previous state (kept or not) reads dev[k]
        torch.cuda.current_stream(self.g.device).wait_event(self.copied[k])
        self.g.unpack(x, out=st["dev"][k])
        self.ready[k].record()
        with torch.cuda.stream(st["stream"]):
            st["stream"].wait_event(self.ready[k])
            st["pin"][k].copy_(st["dev"][k], non_blocking=True)
            self.copied[k].record(st["stream"])
        return k

    def commit(self, k: int) -> None:
        self.futs[k] = self.pool.submit(self._land, k, self.n)
        self.n += 1

    def discard(self, k: int) -> None:
        """The staged state is not kept (the buffer is free once its copy has run)."""

    def save(self, x: torch.Tensor) -> None:
        self.commit(self.stage(x))

    def _copy(self, dst: torch.Tensor, src: torch.Tensor) -> None:
        nbytes = src.numel() * src.element_size()
        per = -(-nbytes // self.COPY_THREADS)                 # ceil(nbytes / threads), rounded up to pages
        step = (per + 4095) // 4096 * 4096 if nbytes > (1 << 20) else nbytes
        d, s = dst.data_ptr(), src.data_ptr()
        futs = [self.copy_pool.submit(ctypes.memmove, d + off, s + off, min(step, nbytes - off))
                for off in range(0, nbytes, max(step, 1))]
        for f in futs:
            f.result()

    def _land(self, k: int, row: int) -> None:
        ev = self.copied[k]
        while not ev.query():            # coarse polling: each wake-up takes the GIL from the stepping thread
            time.sleep(5e-4)
        if row < self.rows.shape[0]:
            self._copy(self.rows[row], self.st["pin"][k])
        else:
            t = torch.empty_like(self.st["pin"][k], device="cpu")
            self._copy(t, self.st["pin"][k])
            with self.lock:
                self.extra.append((row, t))

    def result(self) -> torch.Tensor:
        """(n_saved, n_state) host tensor."""
        for f in self.futs:
            if f is not None:
                f.result()
        torch.cuda.current_stream(self.g.device).synchronize()
        self.st["stream"].synchronize()
        self.pool.shutdown(wait=True)
        self.copy_pool.shutdown(wait=True)
        if not self.extra and self.n == self.rows.shape[0]:
            return self.rows
        more = [t for _, t in sorted(self.extra, key=lambda e: e[0])]
        return torch.cat([self.rows[:min(self.n, self.rows.shape[0])]] + [t[None] for t in more], dim=0)


def _field_at(eval_u, t, params, idx) -> L.Field:
    u = eval_u(t, None)
    bx, by, bz = field_scalars_from_vectors(u, params, idx) if hasattr(u, "Bz") else tuple(u)
    return L.Field(bx, by, bz, 1.0, 0.5, 1.0, 0, 1)


def _add_counts(tot: dict, st: dict) -> None:
    for k in tot:
        tot[k] = max(tot[k], st[k]) if k == "max_krylov" else tot[k] + (1 if k == "kernel_launches" else st[k])


def _check_step(rc: int, t: float, cur: float, t_stop: float, dt_min: float) -> None:
    """The integrator's failures as the reference reports them
    (integrators.py:186-197); other device statuses as TDGLError."""
    if rc == L.TDGL_ENOCONV:
        raise RuntimeError(f"Newton did not converge at t={t:.6e} with dt={min(cur, t_stop - t):.3e}.")
    if rc == L.TDGL_EDTMIN:
        raise RuntimeError(f"dt reduced below dt_min={dt_min:.1e} at t={t:.6e}; aborting.")
    L.check(rc, "tdgl_trap_run")


def _clock_after(t: float, dt: float, t_stop: float, n: int) -> float:
    """The clock after n accepted steps of min(dt, t_stop - t) (no retries)."""
    for _ in range(n):
        if not t < t_stop - 1e-14:
            break
        t += min(dt, t_stop - t)
    return t


def _trap_queued(g, x, t, cur, t_stop, dt, save_every, opts, field, hist, times, tot, dt_min, verbose):
    """The step loop of trapezoidal with the next launch queued on the device
    before the previous one is collected (tdgl_trap_launch_next continues
    from the clock the previous launch leaves), so the GPU steps on while the
    host reads a launch's counters and lands its state.  Each launch makes up
    to save_every accepted steps; its state is staged right behind it in
    stream order and kept when the reference would save it
    (integrators.py:180-182).  A launch is queued while the clock predicted
    without retries is short of t_stop, and again whenever the queue has run
    dry before t_stop (after dt retries).  Returns (t, dt_cur, steps)."""
    stream = torch.cuda.current_stream(g.device)
    queue = []
    g.trap_launch(x, t, cur, save_every, opts, field, stream)
    queue.append(hist.stage(x))
    t_pred = _clock_after(t, dt, t_stop, save_every)
    step = 0
    while queue:
        if len(queue) < 2 and t_pred < t_stop - 1e-14:
            g.trap_launch_next(x, save_every, opts, field, stream)
            queue.append(hist.stage(x))
            t_pred = _clock_after(t_pred, dt, t_stop, save_every)
        rc, t, cur, st = g.trap_collect()
        k = queue.pop(0)
        _add_counts(tot, st)
        step += st["steps"]
        if rc != L.TDGL_OK:
            while queue:                     # the queued continuation is drained, its result dropped
                g.trap_collect()
                hist.discard(queue.pop(0))
            hist.discard(k)
            _check_step(rc, t, cur, t_stop, dt_min)
        if verbose:
            print(f"  t={t:.4f} steps={step} newton={st['newton_iters']} krylov={st['krylov_iters']}")
        if st["steps"] > 0 and step % save_every == 0:
            times.append(t)
            hist.commit(k)
        else:
            hist.discard(k)
        if not queue and t < t_stop - 1e-14:
            g.trap_launch_next(x, save_every, opts, field, stream)
            queue.append(hist.stage(x))
            t_pred = _clock_after(t, dt, t_stop, save_every)
    return t, cur, step


def trapezoidal(x0, params, idx, eval_u: Callable, t_start: float, t_stop: float, dt: float, *,
                newton_tol_f: float = 1e-3, newton_tol_dx: float = 1e-3, newton_max_iter: int = 20,
                tol_gcr: float = 1e-4, eps_mf: float = 1e-4, save_every: int = 1, adaptive: bool = True,
                dt_min: float = 1e-8, progress: bool = True, verbose: bool = False, material=None,
                precision: str = "fp64", jvp: Optional[str] = None, kmax: int = DEFAULT_KMAX,
                krylov: Optional[str] = None, stats: Optional[dict] = None):
    """Implicit trapezoidal integration with Newton-GCR and dt/10 retries
    (integrators.py:92-206).  Returns (times, X_history) with X_history of
    shape (n_state, n_saved), as the reference does.

    The step loop, Newton and Krylov iterations and the retries run inside one
    device launch per saved state; the host only stores saved states, and
    with the GMRES executor the next launch is queued before the previous one
    is collected.  With an ``eval_u`` the device cannot evaluate (a Python
    ``field_func``), one launch per step is made with the field evaluated on
    the host at the step's start.
    """
    jvp = jvp or ("fd" if precision == "fp64" else "analytic")
    g = grid_for(params, idx, material, precision, kmax, default_krylov(krylov, jvp))
    ref = g.ref_tensor(x0)
    _check_real_links(ref, params)          # on the device copy
    x = g.pack(ref)
    opts = L.TrapOpts(float(t_stop), float(dt), float(dt_min), float(newton_tol_f), float(newton_tol_dx),
                      float(tol_gcr), float(eps_mf), int(newton_max_iter), 0, int(bool(adaptive)),
                      {"fd": L.TDGL_JVP_FD, "analytic": L.TDGL_JVP_ANALYTIC}[jvp])
    dev_field = eval_u.device_field() if isinstance(eval_u, FieldSchedule) else None
    t, cur = float(t_start), float(dt)
    times = [t]
    nsteps = _count_steps(t_start, t_stop, dt)
    hist = _History(g, 1 + -(-nsteps // max(int(save_every), 1)))
    hist.save(x)
    tot = {"steps": 0, "newton_iters": 0, "krylov_iters": 0, "rhs_evals": 0, "jvp_evals": 0, "rejections": 0,
           "max_krylov": 0, "kernel_launches": 0}
    step = 0
    if dev_field is not None and g.krylov == "gmres" and t < t_stop - 1e-14:
        t, cur, step = _trap_queued(g, x, t, cur, float(t_stop), float(dt), max(int(save_every), 1), opts, dev_field,
                                    hist, times, tot, float(dt_min), verbose)
    while t < t_stop - 1e-14:
        if dev_field is not None:
            rc, t, cur, st = g.trap_run(x, t, cur, int(save_every), opts, dev_field)
        else:
            rc, t, cur, st = g.trap_run(x, t, cur, 1, opts, _field_at(eval_u, t, params, idx))
        _add_counts(tot, st)
        step += st["steps"]
        _check_step(rc, t, cur, t_stop, dt_min)
        if verbose:
            print(f"  t={t:.4f} steps={step} newton={st['newton_iters']} krylov={st['krylov_iters']}")
        if st["steps"] > 0 and step % save_every == 0:
            times.append(t)
            hist.save(x)
        if st["steps"] == 0 and not (t < t_stop - 1e-14):
            break
    if times[-1] < t:
        times.append(t)
        hist.save(x)
    if stats is not None:
        stats.update(tot)
    H = hist.result().T          # (n_state, n_saved), as the reference returns it
    if _is_torch(x0):
        return torch.tensor(times, dtype=torch.float64), H.to(x0.device)
    return np.array(times), H.numpy()


def forward_euler(x0, params, idx, eval_u: Callable, t_start: float, t_stop: float, dt: float, *,
                  save_every: int = 1, progress: bool = True, material=None):
    """Explicit Euler with ceil((t_stop - t_start)/dt) steps of
    min(dt, t_stop - t) (integrators.py:35-89), run on the device."""
    g = grid_for(params, idx, material, "fp64", DEFAULT_KMAX)
    _check_real_links(x0, params)
    n_steps = int(np.ceil((t_stop - t_start) / dt))
    x = g.pack(x0)
    dev_field = eval_u.device_field() if isinstance(eval_u, FieldSchedule) else None
    t = float(t_start)
    times = [t]
    hist = _History(g, 1 + -(-n_steps // max(int(save_every), 1)))
    hist.save(x)
    s = 0
    while s < n_steps:
        if dev_field is not None:
            nxt = min(n_steps, (s // save_every + 1) * save_every)
            t = g.euler_run(x, t, t_stop, dt, nxt - s, dev_field)
            s = nxt
        else:
            t = g.euler_run(x, t, t_stop, dt, 1, _field_at(eval_u, t, params, idx))
            s += 1
        if s % save_every == 0 or s == n_steps:
            times.append(t)
            hist.save(x)
    H = hist.result().T
    if _is_torch(x0):
        return torch.tensor(times, dtype=torch.float64), H.to(x0.device)
    return np.array(times), H.numpy()


def solve(device, t_start: float = 0.0, t_stop: float = 10.0, dt: float = 0.05, method: str = "trapezoidal",
          x0=None, *, save_every: int = 1, progress: bool = True, verbose: bool = False,
          newton_tol_f: float = 1e-3, newton_tol_dx: float = 1e-3, newton_max_iter: int = 20,
          tol_gcr: float = 1e-4, eps_mf: float = 1e-4, adaptive: bool = True, log_metadata: bool = True,
          log_dir="logs", precision: str = "fp64", jvp: Optional[str] = None, kmax: int = DEFAULT_KMAX,
          krylov: Optional[str] = None):
    """Run a simulation and return a :class:`~nanowire_tdgl_b200.solution.Solution`
    (runner.py:40-163)."""
    from .solution import Solution

    params, idx = device.params, device.idx
    material = getattr(device, "material", None)
    if x0 is None:
        x0_arr = StateVector.uniform_superconducting(params).data
        if material is not None:
            x0_arr[: params.n_interior] *= material.interior_sc_mask
    elif isinstance(x0, StateVector) or hasattr(x0, "data") and not _is_torch(x0) and not isinstance(x0, np.ndarray):
        x0_arr = x0.data
    else:
        x0_arr = x0 if _is_torch(x0) else np.asarray(x0, dtype=np.complex128)
    eval_u = FieldSchedule(device.applied_field, params, idx, t_stop)
    run_stats: dict = {}
    t0 = time.perf_counter()
    if method == "euler":
        times, X = forward_euler(x0_arr, params, idx, eval_u, t_start, t_stop, dt, save_every=save_every,
                                 progress=progress, material=material)
    elif method == "trapezoidal":
        times, X = trapezoidal(x0_arr, params, idx, eval_u, t_start, t_stop, dt, newton_tol_f=newton_tol_f,
                               newton_tol_dx=newton_tol_dx, newton_max_iter=newton_max_iter, tol_gcr=tol_gcr,
                               eps_mf=eps_mf, save_every=save_every, adaptive=adaptive, progress=progress,
                               verbose=verbose, material=material, precision=precision, jvp=jvp, kmax=kmax,
                               krylov=krylov, stats=run_stats)
    else:
        raise ValueError(f"Unknown method {method!r}. Use 'euler' or 'trapezoidal'.")
    wall = time.perf_counter() - t0
    meta = None
    if log_metadata:
        meta = {"method": method, "dt": dt, "t_start": t_start, "t_final": t_stop, "wall_time_s": wall,
                "total_steps": int(len(times)), "params": {k: getattr(params, k) for k in
                ("Nx", "Ny", "Nz", "hx", "hy", "hz", "kappa", "periodic_x", "periodic_y", "periodic_z")},
                "newton_tol_f": newton_tol_f, "newton_tol_dx": newton_tol_dx, "tol_gcr": tol_gcr,
                "precision": precision,
                "krylov": default_krylov(krylov, jvp or ("fd" if precision == "fp64" else "analytic")),
                "device_counters": run_stats,
                "gpu": torch.cuda.get_device_name() if torch.cuda.is_available() else None}
        path = Path(log_dir)
        path.mkdir(parents=True, exist_ok=True)
        with open(path / f"run_{datetime.now().strftime('%Y%m%d_%H%M%S')}.json", "w") as fh:
            json.dump(meta, fh, indent=2, default=str)
    return Solution(times=times, states=X, params=params, idx=idx, device=device, metadata=meta)
