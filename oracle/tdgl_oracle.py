"""CPU oracle for the trapezoidal TDGL stepper — TEST INFRASTRUCTURE ONLY.

This module restates, in plain numpy, the arithmetic of the tdgl3d hot path so
that the CUDA path can be checked against it.  It is imported only by
``tests/``, by ``__graft_entry__.smoke()`` (as the checker) and by the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``.  The product
package never imports it.

Parity pin: this restatement is checked against golden vectors produced by the
reference implementation itself (``tests/golden/make_golden.py`` imports
tdgl3d and records ``eval_f``, index maps, solver answers and a 101-step
trapezoidal trajectory; ``tests/test_oracle_golden.py`` compares).

The reference builds scipy CSR matrices on every call; this restatement is
matrix-free: it assembles the boundary-extended full-grid fields as 3-D arrays
indexed [k, j, i] (so ``ravel()`` is the reference's full-grid index
m = i + mj*j + mk*k) and evaluates the same stencil sums by slicing.

Reference lines followed (paths inside the tdgl3d project):
  expand + boundary conditions  src/tdgl3d/physics/rhs.py:43-139
  RHS assembly                  src/tdgl3d/physics/rhs.py:147-239
  operators                     src/tdgl3d/operators/sparse_operators.py:35-317
  TGCR (trapezoidal)            src/tdgl3d/solvers/tgcr.py:96-156
  Newton (trapezoidal)          src/tdgl3d/solvers/newton.py:76-120
  trapezoidal / forward Euler   src/tdgl3d/solvers/integrators.py:35-206
  B field / supercurrent        src/tdgl3d/physics/bfield.py:12-78,
                                src/tdgl3d/physics/current_density.py:14-72,
                                src/tdgl3d/core/solution.py:94-217
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

TAU_RELAX = 0.1  # src/tdgl3d/operators/sparse_operators.py:223


@dataclass
class OracleGrid:
    """Everything the RHS needs, taken from (params, idx, material)."""

    Nx: int
    Ny: int
    Nz: int
    hx: float
    hy: float
    hz: float
    is_3d: bool
    periodic: tuple
    n: int
    shape: tuple                 # full-grid array shape (nk, Ny+1, Nx+1)
    int_sel: tuple               # slices selecting interior nodes of a full array
    perm: np.ndarray             # reference interior order -> [k, j, i] interior C order
    hole: tuple                  # full-grid bool arrays: link zeroed after BCs (x, y, z)
    hole_int: tuple              # interior bool arrays (reference order): dphi/dt := 0
    kappa_int: Optional[np.ndarray]   # kappa at interior nodes, reference order (None: uniform)
    kappa: float
    sc_int: Optional[np.ndarray]      # interior sc mask, reference order (None: no material)


def make_grid(params, idx, material=None) -> OracleGrid:
    """Collect grid data from reference-compatible objects (duck-typed)."""
    Nx, Ny, Nz = int(params.Nx), int(params.Ny), int(params.Nz)
    is_3d = Nz > 1
    nk = Nz + 1 if is_3d else 1
    shape = (nk, Ny + 1, Nx + 1)
    nx, ny, nz = Nx - 1, Ny - 1, (Nz - 1 if is_3d else 1)
    n = nx * ny * nz
    int_sel = (slice(1, Nz) if is_3d else slice(0, 1), slice(1, Ny), slice(1, Nx))
    # interior_to_full lists nodes with k fastest, i slowest; the [k, j, i]
    # interior block in C order has i fastest.  perm maps one to the other.
    ref = np.arange(n).reshape(nx, ny, nz)           # ref[i, j, k] = reference index
    perm = ref.transpose(2, 1, 0).ravel()             # C order over [k, j, i]
    mfull = np.asarray(idx.interior_to_full)
    expect = np.zeros(shape, dtype=bool).ravel()
    assert mfull.size == n
    holes, holes_int = [], []
    for ax in ("x", "y", "z"):
        h = np.zeros(int(np.prod(shape)), dtype=bool)
        links = np.asarray(getattr(idx, f"hole_{ax}_bc_mask", np.array([], dtype=np.intp)), dtype=np.intp)
        if links.size and (ax != "z" or is_3d):
            h[links] = True
        holes.append(h.reshape(shape))
        hi = np.zeros(n, dtype=bool)
        li = np.asarray(getattr(idx, f"hole_{ax}_bc_interior", np.array([], dtype=np.intp)), dtype=np.intp)
        if li.size and (ax != "z" or is_3d):
            hi[li] = True
        holes_int.append(hi)
    del expect
    kappa_int = None
    sc_int = None
    if material is not None:
        kappa_int = np.asarray(material.kappa, dtype=np.float64)[mfull]
        sc_int = np.asarray(material.interior_sc_mask, dtype=np.float64)
    return OracleGrid(Nx, Ny, Nz, float(params.hx), float(params.hy), float(params.hz), is_3d,
                      (bool(params.periodic_x), bool(params.periodic_y), bool(params.periodic_z)),
                      n, shape, int_sel, perm, tuple(holes), tuple(holes_int), kappa_int,
                      float(params.kappa), sc_int)


# ---------------------------------------------------------------------------
# Full-grid fields with boundary conditions
# ---------------------------------------------------------------------------

def _to_full(g: OracleGrid, v_ref: np.ndarray, dtype) -> np.ndarray:
    """Scatter an interior vector (reference order) into a zero full grid."""
    full = np.zeros(g.shape, dtype=dtype)
    nx, ny = g.Nx - 1, g.Ny - 1
    nz = g.Nz - 1 if g.is_3d else 1
    full[g.int_sel] = v_ref.reshape(nx, ny, nz).transpose(2, 1, 0)
    return full


def _interior(g: OracleGrid, full: np.ndarray) -> np.ndarray:
    """Gather the interior block of a full-grid array in reference order."""
    return full[g.int_sel].transpose(2, 1, 0).reshape(-1)


def boundary_fields(g: OracleGrid, X: np.ndarray, bx: float, by: float, bz: float):
    """Return full-grid (psi, phix, phiy, phiz) after the reference's boundary
    procedure (src/tdgl3d/physics/rhs.py:54-139), in its order:

    1. zero the normal link on planes 0 and N-1 of its own axis;
    2. snapshot; 3. x, y, (z) face writes from the snapshot (zero-current
       Peierls copies of psi, applied-field offsets of the tangential links,
       or periodic wrap-around); edges and corners stay zero;
    4. zero hole-boundary links last.
    The link fields are returned as real arrays (their imaginary part is
    exactly zero in the reference)."""
    n = g.n
    psi = _to_full(g, X[:n], np.complex128)
    fx = _to_full(g, X[n:2 * n].real, np.float64)
    fy = _to_full(g, X[2 * n:3 * n].real, np.float64)
    fz = _to_full(g, X[3 * n:4 * n].real, np.float64) if g.is_3d else np.zeros(g.shape)
    Nx, Ny, Nz = g.Nx, g.Ny, g.Nz
    fx[:, :, [0, Nx - 1]] = 0.0
    fy[:, [0, Ny - 1], :] = 0.0
    if g.is_3d:
        fz[[0, Nz - 1], :, :] = 0.0
    p0, x0, y0, z0 = psi.copy(), fx.copy(), fy.copy(), fz.copy()
    hx, hy, hz = g.hx, g.hy, g.hz
    czxy = bz * hx * hy      # Bz * hx * hy
    cyzx = by * hz * hx      # By * hz * hx
    cxyz = bx * hy * hz      # Bx * hy * hz
    kk = slice(1, Nz) if g.is_3d else slice(0, 1)
    jj, ii = slice(1, Ny), slice(1, Nx)
    # x faces (inner j, k)
    if g.periodic[0]:
        psi[kk, jj, 0] += p0[kk, jj, Nx - 1]
        psi[kk, jj, Nx] += p0[kk, jj, 1]
        fx[kk, jj, 0] += x0[kk, jj, Nx - 1]
        fx[kk, jj, Nx] += x0[kk, jj, 1]
    else:
        psi[kk, jj, 0] += p0[kk, jj, 1] * np.exp(-1j * x0[kk, jj, 0])
        psi[kk, jj, Nx] += p0[kk, jj, Nx - 1] * np.exp(1j * x0[kk, jj, Nx - 1])
        fy[kk, jj, 0] += -czxy + y0[kk, jj, 1]
        fy[kk, jj, Nx] += czxy + y0[kk, jj, Nx - 1]
        fz[kk, jj, 0] += cyzx + z0[kk, jj, 1]
        fz[kk, jj, Nx] += -cyzx + z0[kk, jj, Nx - 1]
    # y faces (inner i, k)
    if g.periodic[1]:
        psi[kk, 0, ii] += p0[kk, Ny - 1, ii]
        psi[kk, Ny, ii] += p0[kk, 1, ii]
        fy[kk, 0, ii] += y0[kk, Ny - 1, ii]
        fy[kk, Ny, ii] += y0[kk, 1, ii]
    else:
        psi[kk, 0, ii] += p0[kk, 1, ii] * np.exp(-1j * y0[kk, 0, ii])
        psi[kk, Ny, ii] += p0[kk, Ny - 1, ii] * np.exp(1j * y0[kk, Ny - 1, ii])
        fx[kk, 0, ii] += czxy + x0[kk, 1, ii]
        fx[kk, Ny, ii] += -czxy + x0[kk, Ny - 1, ii]
        fz[kk, 0, ii] += -cxyz + z0[kk, 1, ii]
        fz[kk, Ny, ii] += cxyz + z0[kk, Ny - 1, ii]
    # z faces (inner i, j), 3-D only
    if g.is_3d:
        if g.periodic[2]:
            psi[0, jj, ii] += p0[Nz - 1, jj, ii]
            psi[Nz, jj, ii] += p0[1, jj, ii]
            fz[0, jj, ii] += z0[Nz - 1, jj, ii]
            fz[Nz, jj, ii] += z0[1, jj, ii]
        else:
            psi[0, jj, ii] += p0[1, jj, ii] * np.exp(-1j * z0[0, jj, ii])
            psi[Nz, jj, ii] += p0[Nz - 1, jj, ii] * np.exp(1j * z0[Nz - 1, jj, ii])
            fx[0, jj, ii] += -cyzx + x0[1, jj, ii]
            fx[Nz, jj, ii] += cyzx + x0[Nz - 1, jj, ii]
            fy[0, jj, ii] += cxyz + y0[1, jj, ii]
            fy[Nz, jj, ii] += -cxyz + y0[Nz - 1, jj, ii]
    fx[g.hole[0]] = 0.0
    fy[g.hole[1]] = 0.0
    if g.is_3d:
        fz[g.hole[2]] = 0.0
    return psi, fx, fy, fz


def _sh(a: np.ndarray, dk: int, dj: int, di: int) -> np.ndarray:
    """a[k+dk, j+dj, i+di] over the interior block (neighbour access)."""
    return a[_shift_sel(a.shape, dk, dj, di)]


def _shift_sel(shape, dk, dj, di):
    nk, nj, ni = shape
    ks = slice(1 + dk, nk - 1 + dk) if nk > 1 else slice(0, 1)
    return (ks, slice(1 + dj, nj - 1 + dj), slice(1 + di, ni - 1 + di))


def eval_f(X: np.ndarray, g: OracleGrid, bx: float = 0.0, by: float = 0.0, bz: float = 0.0) -> np.ndarray:
    """dX/dt at interior nodes, reference order (src/tdgl3d/physics/rhs.py:147-239).

    psi:  sum_d [e^{-i phi_d(m-d)} psi(m-d) - 2 psi(m) + e^{i phi_d(m)} psi(m+d)] / h_d^2
          + sc (1-|psi|^2) psi - (1-sc) psi / 0.1          (GL term only without material)
    phi_a: (sum over the two other Laplacians' stencils, src/tdgl3d/physics/rhs.py:223-225)
          + Im[e^{-i phi_a(m)} conj(psi(m)) psi(m+a)]
          + sum_{b != a} c_b (-phi_b(m+a) + phi_b(m) + phi_b(m+a-b) - phi_b(m-b))
    with c_b = kappa(m)^2 / h_b^2, then zero at interior hole-boundary links.
    """
    psi, fx, fy, fz = boundary_fields(g, X, bx, by, bz)
    hx, hy, hz = g.hx, g.hy, g.hz
    d3 = g.is_3d
    c = _sh(psi, 0, 0, 0)
    # gauge-covariant Laplacian of psi
    Lx = np.exp(-1j * _sh(fx, 0, 0, -1)) * _sh(psi, 0, 0, -1) - 2.0 * c + np.exp(1j * _sh(fx, 0, 0, 0)) * _sh(psi, 0, 0, 1)
    Ly = np.exp(-1j * _sh(fy, 0, -1, 0)) * _sh(psi, 0, -1, 0) - 2.0 * c + np.exp(1j * _sh(fy, 0, 0, 0)) * _sh(psi, 0, 1, 0)
    dpsi = Lx / hx ** 2 + Ly / hy ** 2
    if d3:
        Lz = np.exp(-1j * _sh(fz, -1, 0, 0)) * _sh(psi, -1, 0, 0) - 2.0 * c + np.exp(1j * _sh(fz, 0, 0, 0)) * _sh(psi, 1, 0, 0)
        dpsi = dpsi + Lz / hz ** 2
    gl = (1.0 - np.conj(c) * c) * c
    if g.sc_int is not None:
        sc = _to_full(g, g.sc_int, np.float64)[g.int_sel]
        fpsi = sc * gl - (1.0 - sc) * c / TAU_RELAX
    else:
        fpsi = gl
    dpsi = dpsi + fpsi

    if g.kappa_int is not None:
        k2 = _to_full(g, g.kappa_int, np.float64)[g.int_sel] ** 2
    else:
        k2 = np.full(c.shape, g.kappa ** 2)
    cx, cy = k2 / hx ** 2, k2 / hy ** 2
    cz = k2 / hz ** 2 if d3 else np.zeros_like(k2)

    def lap(f, wx, wy, wz):
        out = (-2.0 * (wx + wy + wz)) * _sh(f, 0, 0, 0)
        out = out + wx * (_sh(f, 0, 0, -1) + _sh(f, 0, 0, 1)) + wy * (_sh(f, 0, -1, 0) + _sh(f, 0, 1, 0))
        if d3:
            out = out + wz * (_sh(f, -1, 0, 0) + _sh(f, 1, 0, 0))
        return out

    def sup(f, dk, dj, di):
        return np.imag(np.exp(-1j * _sh(f, 0, 0, 0)) * np.conj(c) * _sh(psi, dk, dj, di))

    def curl(fb, wb, a, b):
        # a = (dk, dj, di) of the own axis, b = offsets of the other axis
        ak, aj, ai = a
        bk, bj, bi = b
        return wb * (-_sh(fb, ak, aj, ai) + _sh(fb, 0, 0, 0) + _sh(fb, ak - bk, aj - bj, ai - bi) - _sh(fb, -bk, -bj, -bi))

    ex, ey, ez = (0, 0, 1), (0, 1, 0), (1, 0, 0)
    dfx = lap(fx, 2 * cx, cy, cz) + sup(fx, *ex) + curl(fy, cy, ex, ey)
    dfy = lap(fy, cx, 2 * cy, cz) + sup(fy, *ey) + curl(fx, cx, ey, ex)
    if d3:
        dfx = dfx + curl(fz, cz, ex, ez)
        dfy = dfy + curl(fz, cz, ey, ez)
        dfz = lap(fz, cx, cy, 2 * cz) + sup(fz, *ez) + curl(fx, cx, ez, ex) + curl(fy, cy, ez, ey)

    def back(a):
        return a.transpose(2, 1, 0).reshape(-1)

    out = [back(dpsi), back(dfx).astype(np.complex128), back(dfy).astype(np.complex128)]
    out[1][g.hole_int[0]] = 0.0
    out[2][g.hole_int[1]] = 0.0
    if d3:
        o3 = back(dfz).astype(np.complex128)
        o3[g.hole_int[2]] = 0.0
        out.append(o3)
    return np.concatenate(out)


def make_rhs(g: OracleGrid, bx=0.0, by=0.0, bz=0.0) -> Callable[[np.ndarray], np.ndarray]:
    return lambda X: eval_f(X, g, bx, by, bz)


# ---------------------------------------------------------------------------
# Solvers (reference algorithms, same control flow and tests)
# ---------------------------------------------------------------------------

def _rdot(a: np.ndarray, b: np.ndarray) -> float:
    """Re <a, b> = Re sum conj(a) b  (np.vdot(...).real in the reference)."""
    return float(np.vdot(a, b).real)


def _axpy(a: float, x: np.ndarray, y: np.ndarray) -> None:
    """y += a x in place (real scalar, complex vectors), via real views."""
    yr = y.view(np.float64)
    xr = x.view(np.float64)
    if yr.size > 4096:
        from scipy.linalg.blas import daxpy
        daxpy(xr, yr, a=a)
    else:
        yr += a * xr


def tgcr_trap(f: Callable, x_lin: np.ndarray, b: np.ndarray, dt: float, tol: float = 1e-4,
              max_iter: Optional[int] = None, eps_mf: float = 1e-4, stats: Optional[dict] = None):
    """GCR for (I - dt/2 J) d = b with a finite-difference J·p and modified
    Gram-Schmidt over all previous directions (src/tdgl3d/solvers/tgcr.py:96-156).
    Returns the solution, or an empty array when the relative residual is
    still above ``tol`` on exit."""
    N = len(b)
    if max_iter is None:
        max_iter = max(N, int(round(0.2 * N)))
    x = np.zeros_like(b)
    r = b.copy()
    r0 = np.linalg.norm(r)
    rn = r0
    if r0 == 0.0:
        return x
    P, AP = [], []
    f_base = f(x_lin)
    xnorm = np.linalg.norm(x_lin)
    k = 0
    while rn / r0 > tol and k < max_iter:
        k += 1
        p = r.copy()
        eps = eps_mf * (1.0 + xnorm) / np.linalg.norm(p)
        ap = p - (dt / 2.0) * ((f(x_lin + eps * p) - f_base) / eps)
        for pj, apj in zip(P, AP):          # modified Gram-Schmidt, updated in place
            beta = _rdot(ap, apj)
            _axpy(-beta, pj, p)
            _axpy(-beta, apj, ap)
        nap = np.linalg.norm(ap)
        if nap < 1e-14:
            break
        ap /= nap
        p /= nap
        P.append(p)
        AP.append(ap)
        alpha = _rdot(r, ap)
        _axpy(alpha, p, x)
        _axpy(-alpha, ap, r)
        rn = np.linalg.norm(r)
    if stats is not None:
        stats["krylov_iters"] = stats.get("krylov_iters", 0) + k
        stats["tgcr_calls"] = stats.get("tgcr_calls", 0) + 1
    if rn > tol * r0:
        return np.array([], dtype=np.complex128)
    return x


def newton_trap(f: Callable, x0: np.ndarray, gamma: np.ndarray, dt: float, *, tol_f=1e-3,
                tol_dx=1e-3, max_iter=20, tol_gcr=1e-4, eps_mf=1e-4, stats=None):
    """Newton on g(x) = x - dt/2 f(x) - gamma; converged when both the
    infinity norms of g (after the update) and of the update are within
    tolerance (src/tdgl3d/solvers/newton.py:76-120)."""
    x = np.array(x0, dtype=np.complex128)
    fx = f(x)
    for k in range(1, max_iter + 1):
        g = x - (dt / 2.0) * fx - gamma
        dx = tgcr_trap(f, x, -g, dt, tol=tol_gcr, eps_mf=eps_mf, stats=stats)
        if dx.size == 0:
            return x, False, k
        x = x + dx
        fx = f(x)
        g = x - (dt / 2.0) * fx - gamma
        if stats is not None:
            stats["newton_iters"] = stats.get("newton_iters", 0) + 1
        if np.linalg.norm(g, np.inf) <= tol_f and np.linalg.norm(dx, np.inf) <= tol_dx:
            return x, True, k
    return x, False, max_iter


def trapezoidal(x0, g: OracleGrid, field: Callable[[float], tuple], t_start, t_stop, dt, *,
                newton_tol_f=1e-3, newton_tol_dx=1e-3, newton_max_iter=20, tol_gcr=1e-4,
                eps_mf=1e-4, save_every=1, adaptive=True, dt_min=1e-8, stats=None,
                max_steps: Optional[int] = None):
    """Trapezoidal stepping with Newton-GCR and dt/10 retries
    (src/tdgl3d/solvers/integrators.py:92-206).  ``field(t)`` returns the
    applied (Bx, By, Bz) at the start of a step.  ``max_steps`` stops early
    after that many accepted steps (used to time a bounded sample)."""
    X = np.array(x0, dtype=np.complex128)
    t = t_start
    cur = dt
    times, hist = [t], [X.copy()]
    step = 0
    while t < t_stop - 1e-14:
        if max_steps is not None and step >= max_steps:
            break
        dta = min(cur, t_stop - t)
        f = make_rhs(g, *field(t))
        fn = f(X)
        x_pred = X + dta * fn
        gamma = X + (dta / 2.0) * fn
        xn, ok, _ = newton_trap(f, x_pred, gamma, dta, tol_f=newton_tol_f, tol_dx=newton_tol_dx,
                                max_iter=newton_max_iter, tol_gcr=tol_gcr, eps_mf=eps_mf, stats=stats)
        if ok:
            X = xn
            t += dta
            step += 1
            if step % save_every == 0:
                times.append(t)
                hist.append(X.copy())
            cur = dt
        else:
            if stats is not None:
                stats["rejections"] = stats.get("rejections", 0) + 1
            if not adaptive:
                raise RuntimeError(f"Newton did not converge at t={t:.6e} with dt={dta:.3e}.")
            cur /= 10.0
            if cur < dt_min:
                raise RuntimeError(f"dt reduced below dt_min={dt_min:.1e} at t={t:.6e}; aborting.")
    if times[-1] < t:
        times.append(t)
        hist.append(X.copy())
    return np.array(times), np.column_stack(hist)


def forward_euler(x0, g: OracleGrid, field: Callable[[float], tuple], t_start, t_stop, dt, *,
                  save_every=1):
    """Explicit Euler with ceil((t_stop-t_start)/dt) steps of min(dt, t_stop-t)
    (src/tdgl3d/solvers/integrators.py:35-89)."""
    n_steps = int(np.ceil((t_stop - t_start) / dt))
    X = np.array(x0, dtype=np.complex128)
    times, hist = [t_start], [X.copy()]
    t = t_start
    for s in range(n_steps):
        dta = min(dt, t_stop - t)
        X = X + dta * eval_f(X, g, *field(t))
        t += dta
        if (s + 1) % save_every == 0 or s == n_steps - 1:
            times.append(t)
            hist.append(X.copy())
    return np.array(times), np.column_stack(hist)


def field_schedule(Bx=0.0, By=0.0, Bz=0.0, t_on_fraction=2.0 / 3.0, ramp=False,
                   ramp_fraction=0.5, t_stop=1.0):
    """B(t) of src/tdgl3d/physics/applied_field.py:42-56 as a closure of t."""
    def fld(t):
        if t <= 0 or t > t_stop * t_on_fraction:
            return 0.0, 0.0, 0.0
        s = 1.0
        if ramp:
            tr = t_stop * ramp_fraction
            s = min(t / tr, 1.0) if tr > 0 else 1.0
        return Bx * s, By * s, Bz * s
    return fld


# ---------------------------------------------------------------------------
# Observables
# ---------------------------------------------------------------------------

def psi_squared(X: np.ndarray, g: OracleGrid) -> np.ndarray:
    """|psi|^2 at interior nodes (src/tdgl3d/core/solution.py:76-78)."""
    return np.abs(X[: g.n]) ** 2


def bfield(X: np.ndarray, g: OracleGrid, bx=0.0, by=0.0, bz=0.0):
    """B = curl(phi) / (h h) at interior nodes from the boundary-extended links
    (src/tdgl3d/core/solution.py:94-158 with src/tdgl3d/physics/bfield.py:12-78)."""
    _, fx, fy, fz = boundary_fields(g, X, bx, by, bz)
    back = lambda a: a.transpose(2, 1, 0).reshape(-1)  # noqa: E731
    Bz = back((_sh(fx, 0, 0, 0) - _sh(fx, 0, 1, 0) - _sh(fy, 0, 0, 0) + _sh(fy, 0, 0, 1)) / (g.hx * g.hy))
    if g.is_3d:
        Bx = back((_sh(fy, 0, 0, 0) - _sh(fy, 1, 0, 0) - _sh(fz, 0, 0, 0) + _sh(fz, 0, 1, 0)) / (g.hy * g.hz))
        By = back((_sh(fz, 0, 0, 0) - _sh(fz, 0, 0, 1) - _sh(fx, 0, 0, 0) + _sh(fx, 1, 0, 0)) / (g.hz * g.hx))
    else:
        Bx = np.zeros(g.n)
        By = np.zeros(g.n)
    return Bx, By, Bz


def supercurrent_density(X: np.ndarray, g: OracleGrid):
    """J_s,d = Im[conj(psi(m)) e^{-i phi_d(m)} psi(m+d)] on the zero-extended
    state, without boundary conditions (src/tdgl3d/core/solution.py:180-217,
    src/tdgl3d/physics/current_density.py:14-72)."""
    n = g.n
    psi = _to_full(g, X[:n], np.complex128)
    fx = _to_full(g, X[n:2 * n].real, np.float64)
    fy = _to_full(g, X[2 * n:3 * n].real, np.float64)
    c = _sh(psi, 0, 0, 0)
    back = lambda a: a.transpose(2, 1, 0).reshape(-1)  # noqa: E731
    Jx = back(np.imag(np.conj(c) * np.exp(-1j * _sh(fx, 0, 0, 0)) * _sh(psi, 0, 0, 1)))
    Jy = back(np.imag(np.conj(c) * np.exp(-1j * _sh(fy, 0, 0, 0)) * _sh(psi, 0, 1, 0)))
    if g.is_3d:
        fz = _to_full(g, X[3 * n:4 * n].real, np.float64)
        Jz = back(np.imag(np.conj(c) * np.exp(-1j * _sh(fz, 0, 0, 0)) * _sh(psi, 1, 0, 0)))
    else:
        Jz = np.zeros(n)
    return Jx, Jy, Jz
