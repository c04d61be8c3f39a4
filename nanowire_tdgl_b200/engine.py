"""Device contexts: one C-ABI context per (grid, holes, material, precision).

A :class:`DeviceGrid` owns the ``tdgl_ctx`` and a few staging tensors; torch
provides the device memory and the CUDA stream, the numerics are the C ABI's.
"""

from __future__ import annotations

import ctypes as C
import weakref
from typing import Optional

import numpy as np
import torch

from . import _lib as L

PRECISIONS = {"fp64": L.TDGL_FP64, "mixed": L.TDGL_MIXED}
JVP_MODES = {"fd": L.TDGL_JVP_FD, "analytic": L.TDGL_JVP_ANALYTIC}
KRYLOV = {"gmres": L.TDGL_KRYLOV_GMRES, "gcr": L.TDGL_KRYLOV_GCR}


def _require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("nanowire_tdgl_b200 needs a CUDA device (B200, sm_100a); none is visible")
    return torch.device("cuda", torch.cuda.current_device())


def stream_handle() -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: Optional[torch.Tensor]) -> C.c_void_p:
    return C.c_void_p(0 if t is None else t.data_ptr())


def _i64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64).ravel())


def descriptors(params, idx, material=None):
    """(GridDesc, MaterialDesc, keep-alive list) for the C ABI from
    reference-compatible params / idx / material objects."""
    is_3d = int(params.Nz) > 1
    g = L.GridDesc(int(params.Nx), int(params.Ny), int(params.Nz), int(bool(params.periodic_x)),
                   int(bool(params.periodic_y)), int(bool(params.periodic_z)), float(params.hx),
                   float(params.hy), float(params.hz), float(params.kappa))
    md = L.MaterialDesc()
    keep = []
    for a, ax in enumerate("xyz"):
        links = _i64(getattr(idx, f"hole_{ax}_bc_mask", []))
        inner = _i64(getattr(idx, f"hole_{ax}_bc_interior", []))
        if ax == "z" and not is_3d:
            links, inner = links[:0], inner[:0]
        keep += [links, inner]
        md.hole_links[a] = links.ctypes.data_as(C.POINTER(C.c_int64))
        md.n_hole_links[a] = links.size
        md.hole_interior[a] = inner.ctypes.data_as(C.POINTER(C.c_int64))
        md.n_hole_interior[a] = inner.size
    if material is not None:
        kap = np.ascontiguousarray(np.asarray(material.kappa, dtype=np.float64))
        sc = np.ascontiguousarray(np.asarray(material.interior_sc_mask, dtype=np.float64))
        if kap.shape != (params.dim_x,) or sc.shape != (params.n_interior,):
            raise ValueError("material arrays do not match the grid")
        keep += [kap, sc]
        md.kappa_full = kap.ctypes.data_as(C.POINTER(C.c_double))
        md.sc_interior = sc.ctypes.data_as(C.POINTER(C.c_double))
    return g, md, keep


class DeviceGrid:
    """Device description of one grid with its holes and material map."""

    def __init__(self, params, idx, material=None, precision: str = "fp64", kmax: int = 64,
                 krylov: str = "gmres"):
        self.lib = L.load()
        self.device = _require_cuda()
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self.params = params
        self.precision = precision
        self.kmax = int(kmax)
        if krylov not in KRYLOV:
            raise ValueError(f"krylov must be one of {sorted(KRYLOV)}")
        self.krylov = krylov
        g, md, keep = descriptors(params, idx, material)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            L.check(self.lib.tdgl_ctx_create(C.byref(g), C.byref(md), PRECISIONS[precision], self.kmax,
                                             C.byref(h)), "tdgl_ctx_create")
        self.handle = h
        L.check(self.lib.tdgl_ctx_set_krylov(h, KRYLOV[krylov]), "tdgl_ctx_set_krylov")
        self.n = int(self.lib.tdgl_n_interior(h))
        self.npad = int(self.lib.tdgl_npad(h))
        self.state_len = int(self.lib.tdgl_state_len(h))
        self.n_state = int(params.n_state)
        self._finalizer = weakref.finalize(self, self.lib.tdgl_ctx_destroy, h)

    # -- buffers ------------------------------------------------------------
    def empty_state(self) -> torch.Tensor:
        return torch.zeros(self.state_len, dtype=torch.float64, device=self.device)

    def ref_tensor(self, X) -> torch.Tensor:
        """Reference-layout complex128 state on the device (copied if needed)."""
        if isinstance(X, torch.Tensor):
            t = X.to(device=self.device, dtype=torch.complex128)
        else:
            a = np.asarray(X)
            if a.dtype != np.complex128:
                a = a.astype(np.complex128)
            t = torch.from_numpy(np.ascontiguousarray(a)).to(self.device, non_blocking=False)
        if t.shape != (self.n_state,):
            raise ValueError(f"State vector length {tuple(t.shape)} does not match expected ({self.n_state},)")
        return t.contiguous()

    def pack(self, X, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Reference layout -> device layout (FP64)."""
        ref = self.ref_tensor(X)
        out = self.empty_state() if out is None else out
        L.check(self.lib.tdgl_pack(self.handle, _ptr(ref), _ptr(out), stream_handle()), "tdgl_pack")
        return out

    def unpack(self, x: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Device layout -> reference layout (complex128 tensor on the device)."""
        out = torch.empty(self.n_state, dtype=torch.complex128, device=self.device) if out is None else out
        L.check(self.lib.tdgl_unpack(self.handle, _ptr(x), _ptr(out), stream_handle()), "tdgl_unpack")
        return out

    # -- operators -----------------------------------------------------------
    def rhs(self, x: torch.Tensor, B=(0.0, 0.0, 0.0), out: Optional[torch.Tensor] = None) -> torch.Tensor:
        out = self.empty_state() if out is None else out
        L.check(self.lib.tdgl_rhs(self.handle, _ptr(x), _ptr(out), *map(float, B), stream_handle()), "tdgl_rhs")
        return out

    def eval_f_ref(self, X, B=(0.0, 0.0, 0.0)) -> torch.Tensor:
        ref = self.ref_tensor(X)
        out = torch.empty_like(ref)
        L.check(self.lib.tdgl_eval_f(self.handle, _ptr(ref), _ptr(out), *map(float, B), stream_handle()),
                "tdgl_eval_f")
        return out

    def jvp(self, x: torch.Tensor, p: torch.Tensor, dt: float, mode: str = "analytic", eps_mf: float = 1e-4,
            B=(0.0, 0.0, 0.0)) -> torch.Tensor:
        """ap = p - dt/2 J(x) p.  mode "fd" / "analytic" (FP64), or "krylov": the
        product as this context's analytic-product Krylov solves compute it
        (FP32 for a mixed-precision context; the step graph's stencil kernel)."""
        out = self.empty_state()
        mid = L.TDGL_JVP_KRYLOV if mode == "krylov" else JVP_MODES[mode]
        L.check(self.lib.tdgl_jvp(self.handle, _ptr(x), _ptr(p), _ptr(out), float(dt), mid,
                                  float(eps_mf), *map(float, B), stream_handle()), "tdgl_jvp")
        return out

    def observables(self, x: torch.Tensor, B=(0.0, 0.0, 0.0)) -> dict:
        outs = [torch.empty(self.n, dtype=torch.float64, device=self.device) for _ in range(7)]
        L.check(self.lib.tdgl_observables(self.handle, _ptr(x), *map(float, B), *[_ptr(o) for o in outs],
                                          stream_handle()), "tdgl_observables")
        return dict(zip(("psi2", "Bx", "By", "Bz", "Jx", "Jy", "Jz"), outs))

    def adjoint_solve(self, x: torch.Tensor, b: torch.Tensor, h: float, tol: float, B=(0.0, 0.0, 0.0)):
        """(I - h J(x)^T) mu = b on the device (FP64 context): (mu, iterations,
        converged); at kmax iterations without convergence, mu is the last
        iterate."""
        mu = self.empty_state()
        it = C.c_int32(0)
        rc = self.lib.tdgl_adjoint_solve(self.handle, _ptr(x), _ptr(b), _ptr(mu), float(h), float(tol),
                                         *map(float, B), C.byref(it), stream_handle())
        if rc not in (L.TDGL_OK, L.TDGL_ENOCONV):
            L.check(rc, "tdgl_adjoint_solve")
        return mu, int(it.value), rc == L.TDGL_OK

    def plaquette_winding(self, x: torch.Tensor, mask_threshold: float) -> torch.Tensor:
        """Winding numbers of all plaquettes: (slices, Nx-2, Ny-2), NaN where masked."""
        p = self.params
        ns = max(p.Nz - 1, 1)
        w = torch.empty((ns, p.Nx - 2, p.Ny - 2), dtype=torch.float64, device=self.device)
        L.check(self.lib.tdgl_plaquette_winding(self.handle, _ptr(x), float(mask_threshold), _ptr(w),
                                                stream_handle()), "tdgl_plaquette_winding")
        return w

    def convergence_means(self, x: torch.Tensor, sc_ref: Optional[torch.Tensor] = None) -> torch.Tensor:
        """[mean |psi|^2, mean |J_s|, count] over nodes with sc_ref > 0 (all without)."""
        out = torch.empty(3, dtype=torch.float64, device=self.device)
        L.check(self.lib.tdgl_convergence_means(self.handle, _ptr(x), _ptr(sc_ref) if sc_ref is not None else None,
                                                _ptr(out), stream_handle()), "tdgl_convergence_means")
        return out

    # -- solvers --------------------------------------------------------------
    def tgcr(self, x_lin: torch.Tensor, b: torch.Tensor, dt: float, tol: float, max_iter: int, eps_mf: float,
             jvp: str, B) -> tuple[Optional[torch.Tensor], dict]:
        d = self.empty_state()
        st = L.Stats()
        rc = self.lib.tdgl_tgcr_trap(self.handle, _ptr(x_lin), _ptr(b), _ptr(d), float(dt), float(tol),
                                     int(max_iter), float(eps_mf), JVP_MODES[jvp], *map(float, B), C.byref(st),
                                     stream_handle())
        if rc == L.TDGL_ENOCONV:
            return None, st.as_dict()
        L.check(rc, "tdgl_tgcr_trap")
        return d, st.as_dict()

    def newton(self, x: torch.Tensor, gamma: torch.Tensor, dt: float, tol_f: float, tol_dx: float,
               max_iter: int, tol_gcr: float, eps_mf: float, jvp: str, B) -> dict:
        st = L.Stats()
        rc = self.lib.tdgl_newton_trap(self.handle, _ptr(x), _ptr(gamma), float(dt), float(tol_f), float(tol_dx),
                                       int(max_iter), float(tol_gcr), float(eps_mf), JVP_MODES[jvp],
                                       *map(float, B), C.byref(st), stream_handle())
        L.check(rc, "tdgl_newton_trap")
        return st.as_dict()

    def trap_run(self, x: torch.Tensor, t: float, dt_cur: float, max_steps: int, opts: L.TrapOpts,
                 field: L.Field) -> tuple[int, float, float, dict]:
        tt, dd = C.c_double(t), C.c_double(dt_cur)
        st = L.Stats()
        rc = self.lib.tdgl_trap_run(self.handle, _ptr(x), C.byref(tt), C.byref(dd), int(max_steps), C.byref(opts),
                                    C.byref(field), C.byref(st), stream_handle())
        return rc, tt.value, dd.value, st.as_dict()

    def vjp(self, x: torch.Tensor, v: torch.Tensor, B=(0.0, 0.0, 0.0), want_sc: bool = True):
        """Adjoint of :meth:`rhs` at x (device layout): returns (J^T v,
        d(v.f)/d sc per node [device order, or None], d(v.f)/d kappa^2 per node,
        d(v.f)/d(Bx, By, Bz, kappa))."""
        gx = torch.empty_like(x)
        gsc = torch.empty(self.n, dtype=torch.float64, device=self.device) if want_sc else None
        gk2 = torch.empty(self.n, dtype=torch.float64, device=self.device)
        gpar = torch.empty(4, dtype=torch.float64, device=self.device)
        L.check(self.lib.tdgl_vjp(self.handle, _ptr(x), _ptr(v), *map(float, B), _ptr(gx), _ptr(gsc), _ptr(gk2),
                                  _ptr(gpar), stream_handle()), "tdgl_vjp")
        return gx, gsc, gk2, gpar

    KERNEL_TYPES = ("prepare", "predict", "newton_rhs", "stencil", "projections", "orthogonalisation", "update",
                    "accept", "arnoldi_product", "arnoldi_orthogonalisation", "arnoldi_projections")

    def kernel_timers(self) -> dict:
        """Per-kernel-type device time of the graph executor's launches so far
        (needs TDGL_PROFILE set when the solver workspace was created)."""
        buf = (C.c_uint64 * 32)()
        L.check(self.lib.tdgl_profile(self.handle, buf, 32, 0), "tdgl_profile")
        return {name: {"ms": buf[k] / 1e6, "launches": int(buf[16 + k])} for k, name in enumerate(self.KERNEL_TYPES)}

    def trap_launch(self, x: torch.Tensor, t: float, dt_cur: float, max_steps: int, opts: L.TrapOpts,
                    field: L.Field, stream: torch.cuda.Stream) -> None:
        """Enqueue up to max_steps steps on ``stream`` (returns at once)."""
        L.check(self.lib.tdgl_trap_launch(self.handle, _ptr(x), float(t), float(dt_cur), int(max_steps),
                                          C.byref(opts), C.byref(field), C.c_void_p(stream.cuda_stream)),
                "tdgl_trap_launch")

    def trap_launch_next(self, x: torch.Tensor, max_steps: int, opts: L.TrapOpts, field: L.Field,
                         stream: torch.cuda.Stream) -> None:
        """Enqueue up to max_steps more steps continuing from the clock and state
        the previous launch leaves on the device (returns at once)."""
        L.check(self.lib.tdgl_trap_launch_next(self.handle, _ptr(x), int(max_steps), C.byref(opts), C.byref(field),
                                               C.c_void_p(stream.cuda_stream)), "tdgl_trap_launch_next")

    def trap_collect(self) -> tuple[int, float, float, dict]:
        """Results of the oldest queued launch (waits for it)."""
        tt, dd = C.c_double(0.0), C.c_double(0.0)
        st = L.Stats()
        rc = self.lib.tdgl_trap_collect(self.handle, C.byref(tt), C.byref(dd), C.byref(st))
        return rc, tt.value, dd.value, st.as_dict()

    def set_blocks(self, stream_blocks: int, krylov_blocks: int, fused: int = -1) -> None:
        """Block counts of the step graph's grid-stride and Arnoldi kernels, and
        the Arnoldi product and projections as one kernel (1), two (0) or the
        default (-1)."""
        L.check(self.lib.tdgl_ctx_set_blocks(self.handle, int(stream_blocks), int(krylov_blocks), int(fused)),
                "tdgl_ctx_set_blocks")

    def set_poly(self, degree: int) -> None:
        """Degree of the polynomial preconditioner of the analytic-product GMRES
        solves (0 off, -1 the default)."""
        L.check(self.lib.tdgl_ctx_set_poly(self.handle, int(degree)), "tdgl_ctx_set_poly")

    def set_limits(self, wait_ns: int = 0, loop_cap: int = 0) -> None:
        """Limits of the device's bounded waits (ns) and of one step-graph
        launch's loop iterations; 0 restores the default."""
        L.check(self.lib.tdgl_ctx_set_limits(self.handle, int(wait_ns), int(loop_cap)), "tdgl_ctx_set_limits")

    @property
    def poly_degree(self) -> int:
        return int(self.lib.tdgl_ctx_poly_degree(self.handle))

    def euler_run(self, x: torch.Tensor, t: float, t_stop: float, dt: float, n_steps: int, field: L.Field) -> float:
        tt = C.c_double(t)
        L.check(self.lib.tdgl_euler_run(self.handle, _ptr(x), C.byref(tt), float(t_stop), float(dt), int(n_steps),
                                        C.byref(field), stream_handle()), "tdgl_euler_run")
        return tt.value


_CACHE: dict = {}
_WEIGHTS: dict = {}


def _fingerprint(a: np.ndarray) -> int:
    """64-bit fingerprint of an array's bytes (for the context cache key): the
    sum, modulo 2^64, of its 8-byte words times odd position-dependent weights,
    so that a changed or moved entry changes it (a vectorised pass, several
    times faster than hashing a byte copy of the array)."""
    b = np.ascontiguousarray(a).reshape(-1).view(np.uint8)
    pad = (-b.size) % 8
    if pad:
        b = np.concatenate([b, np.zeros(pad, np.uint8)])
    w = b.view(np.uint64)
    wt = _WEIGHTS.get(w.size)
    if wt is None:
        wt = (np.arange(w.size, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)) | np.uint64(1)
        if len(_WEIGHTS) > 32:
            _WEIGHTS.clear()
        _WEIGHTS[w.size] = wt
    with np.errstate(over="ignore"):
        return int(np.add.reduce(w * wt, dtype=np.uint64))


def grid_for(params, idx, material=None, precision: str = "fp64", kmax: int = 64,
             krylov: str = "gmres") -> DeviceGrid:
    """Cached :class:`DeviceGrid` for these objects (keyed by identity and by
    the hole / material contents, so a device modified after first use is
    rebuilt)."""
    def sig(a):
        a = np.asarray(a)
        return (a.shape, a.dtype.str, _fingerprint(a)) if a.size else (a.shape, 0)
    key = (id(params), id(idx), id(material), precision, int(kmax), krylov,
           (params.Nx, params.Ny, params.Nz, params.hx, params.hy, params.hz, params.kappa,
            bool(params.periodic_x), bool(params.periodic_y), bool(params.periodic_z)),
           tuple(sig(getattr(idx, f"hole_{a}_bc_mask", [])) for a in "xyz"),
           tuple(sig(getattr(idx, f"hole_{a}_bc_interior", [])) for a in "xyz"),
           None if material is None else (sig(material.kappa), sig(material.interior_sc_mask)))
    g = _CACHE.get(key)
    if g is None:
        if len(_CACHE) > 16:
            _CACHE.clear()
        g = DeviceGrid(params, idx, material, precision, kmax, krylov)
        _CACHE[key] = g
    return g
