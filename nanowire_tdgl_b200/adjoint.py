"""Differentiation form: gradients through the trapezoidal stepper.

The reference has no derivatives; this module adds them on top of the device
stepper and the hand-written adjoint of the RHS (``tdgl_vjp``).

Discrete adjoint of one trapezoidal step (src/tdgl3d/solvers/
integrators.py:150-197): x_{n+1} solves

    G(x_{n+1}; x_n, theta) = x_{n+1} - dt/2 f(x_{n+1}) - x_n - dt/2 f(x_n) = 0,

with the applied field held at its value at t_n.  For lambda = dL/dx_{n+1},

    (I - dt/2 J(x_{n+1}))^T mu = lambda,
    dL/dx_n   = mu + dt/2 J(x_n)^T mu,
    dL/dtheta += dt/2 mu^T (df/dtheta(x_{n+1}) + df/dtheta(x_n)),

for theta = the superconducting mask sc (sc = 1 - s for a suppression field
s), the applied field (Bx, By, Bz) and a uniform kappa.  The forward pass
keeps the state every ``checkpoint_every`` steps; the backward pass
recomputes each segment from its checkpoint with the same (deterministic)
stepper, then walks it in reverse.  Transposed solves use restarted GMRES in
FP64 on the device with J^T products from the adjoint kernel.

State layouts: the "real" layout of this module is [psi_re, psi_im, phi_x,
phi_y, (phi_z)], each of n_interior entries in the reference's interior order.
"""

from __future__ import annotations

import math
from typing import Callable, Optional

import numpy as np
import torch

from . import _lib as L
from .engine import grid_for


def real_to_device(grid, xr: torch.Tensor) -> torch.Tensor:
    """Real layout -> device layout (FP64)."""
    n = grid.n
    nc = xr.numel() // n
    parts = [torch.complex(xr[:n], xr[n:2 * n])]
    parts += [xr[c * n:(c + 1) * n].to(torch.complex128) for c in range(2, nc)]
    return grid.pack(torch.cat(parts).to(grid.device))


def device_to_real(grid, xd: torch.Tensor) -> torch.Tensor:
    """Device layout -> real layout."""
    ref = grid.unpack(xd)
    n = grid.n
    nc = ref.numel() // n + 1
    parts = [ref[:n].real, ref[:n].imag] + [ref[c * n:(c + 1) * n].real for c in range(1, nc - 1)]
    return torch.cat(parts)


def node_to_reference_order(grid, a: torch.Tensor) -> torch.Tensor:
    """Per-node array in device order -> the reference's interior order."""
    v = grid.empty_state()
    v[:grid.n] = a
    return grid.unpack(v).real[:grid.n].clone()


class _RHS(torch.autograd.Function):
    """f(x; B) on the device; backward through the hand-written adjoint kernel."""

    @staticmethod
    def forward(ctx, xr, bx, by, bz, grid):
        B = (float(bx), float(by), float(bz))
        xd = real_to_device(grid, xr.detach().to(torch.float64))
        fd = grid.rhs(xd, B)
        ctx.save_for_backward(xd)
        ctx.grid, ctx.B = grid, B
        ctx.bdev = [b.device for b in (bx, by, bz)]
        return device_to_real(grid, fd).to(xr.device)

    @staticmethod
    def backward(ctx, gout):
        (xd,) = ctx.saved_tensors
        grid = ctx.grid
        vd = real_to_device(grid, gout.detach().to(torch.float64).contiguous())
        gx, _, _, gpar = grid.vjp(xd, vd, ctx.B, want_sc=False)
        gxr = device_to_real(grid, gx).to(gout.device)
        return gxr, gpar[0].to(ctx.bdev[0]), gpar[1].to(ctx.bdev[1]), gpar[2].to(ctx.bdev[2]), None


def rhs(xr: torch.Tensor, params, idx, material=None, B=(0.0, 0.0, 0.0)) -> torch.Tensor:
    """Differentiable eval_f (src/tdgl3d/physics/rhs.py:147-239) in the real
    layout: forward on the device in FP64, backward by the adjoint kernel.
    ``B`` entries may be 0-d tensors that require gradients."""
    grid = grid_for(params, idx, material, "fp64", 8)
    bt = [b if isinstance(b, torch.Tensor) else torch.tensor(float(b), dtype=torch.float64) for b in B]
    return _RHS.apply(xr, bt[0], bt[1], bt[2], grid)


def _gmres(matvec: Callable[[torch.Tensor], torch.Tensor], b: torch.Tensor, tol: float, restart: int = 60,
           max_restarts: int = 20, x0: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Restarted GMRES for A x = b in FP64 on the device, from x0 (zero by
    default), to ||b - A x|| <= tol ||b||.  The basis is one (restart + 1) x n
    matrix; each iteration orthogonalises with classical Gram-Schmidt applied
    twice (as stable as the modified form), each pass one matrix-vector
    product for the projections and one for the update, and moves only the
    new Hessenberg column to the host for the Givens rotations."""
    x = torch.zeros_like(b) if x0 is None else x0.clone()
    bn = float(torch.linalg.vector_norm(b))
    if bn == 0.0:
        return torch.zeros_like(b)
    n = b.numel()
    V = torch.empty((restart + 1, n), dtype=b.dtype, device=b.device)
    for cycle in range(max_restarts):
        r = b.clone() if x0 is None and cycle == 0 else b - matvec(x)
        beta = float(torch.linalg.vector_norm(r))
        if beta <= tol * bn:
            return x
        V[0] = r / beta
        H = np.zeros((restart + 1, restart))
        cs, sn = np.zeros(restart), np.zeros(restart)
        gv = np.zeros(restart + 1)
        gv[0] = beta
        k_done = 0
        for k in range(restart):
            w = matvec(V[k])
            Vk = V[:k + 1]
            h = torch.mv(Vk, w)
            w = w - torch.mv(Vk.t(), h)
            h2 = torch.mv(Vk, w)
            w = w - torch.mv(Vk.t(), h2)
            col = torch.cat([h + h2, torch.linalg.vector_norm(w)[None]]).cpu().numpy()
            H[:k + 2, k] = col
            for i in range(k):
                a_, b_ = H[i, k], H[i + 1, k]
                H[i, k] = cs[i] * a_ + sn[i] * b_
                H[i + 1, k] = -sn[i] * a_ + cs[i] * b_
            r_ = math.hypot(H[k, k], H[k + 1, k])
            cs[k], sn[k] = (H[k, k] / r_, H[k + 1, k] / r_) if r_ > 0 else (1.0, 0.0)
            H[k, k], H[k + 1, k] = r_, 0.0
            gv[k + 1] = -sn[k] * gv[k]
            gv[k] = cs[k] * gv[k]
            k_done = k + 1
            if abs(gv[k + 1]) <= tol * bn or H[k, k] == 0.0 or col[-1] == 0.0:
                break
            V[k + 1] = w / float(col[-1])
        y = np.linalg.solve(np.triu(H[:k_done, :k_done]), gv[:k_done])
        x = x + torch.mv(V[:k_done].t(), torch.as_tensor(y, dtype=b.dtype, device=b.device))
    return x


def trapezoidal_gradient(x0, params, idx, t_start: float, t_stop: float, dt: float,
                         loss: Callable[[torch.Tensor], torch.Tensor], *, material=None, B=(0.0, 0.0, 0.0),
                         checkpoint_every: int = 50, precision: str = "fp64", newton_tol_f: float = 1e-8,
                         newton_tol_dx: float = 1e-3, newton_max_iter: int = 20, tol_gcr: float = 1e-6,
                         eps_mf: float = 1e-4, kmax: int = 64, adaptive: bool = True, dt_min: float = 1e-8,
                         adjoint_tol: float = 1e-10, backward: bool = True) -> dict:
    """Run the trapezoidal stepper from x0 (reference complex128 layout) over
    [t_start, t_stop] with the constant field B, evaluate loss(x_final) (x in
    the real layout, a torch tensor on the device) and return its gradients:

    ``loss`` (float), ``x_final`` (device layout), ``grad_x0`` (real layout),
    ``grad_sc`` (reference interior order; None without a material map; the
    gradient with respect to a suppression field s = 1 - sc is its negative),
    ``grad_B`` (Bx, By, Bz), ``grad_kappa`` (uniform kappa; 0 with per-node
    kappa), ``steps``, ``adjoint_iters``.  With ``backward=False`` only the
    forward pass runs (``loss``, ``x_final``, ``steps``).
    """
    grid = grid_for(params, idx, material, precision, kmax)
    jvp = L.TDGL_JVP_ANALYTIC
    opts = L.TrapOpts(float(t_stop), float(dt), float(dt_min), float(newton_tol_f), float(newton_tol_dx),
                      float(tol_gcr), float(eps_mf), int(newton_max_iter), 0, int(bool(adaptive)), jvp)
    fld = L.Field(float(B[0]), float(B[1]), float(B[2]), 1.0, 0.0, float(t_stop), 0, 1)
    C = max(int(checkpoint_every), 1)

    def step(x, t, cur):
        rc, t2, cur2, st = grid.trap_run(x, t, cur, 1, opts, fld)
        L.check(rc, "tdgl_trap_run")
        if st["steps"] != 1:
            raise RuntimeError(f"trapezoidal step did not advance at t={t:.6e}")
        return t2, cur2

    # forward with checkpoints
    x = grid.pack(x0)
    t, cur = float(t_start), float(dt)
    ckpt = {0: (x.clone(), t, cur)}
    dts = []
    while t < t_stop - 1e-14:
        t0 = t
        t, cur = step(x, t, cur)
        dts.append(t - t0)
        if len(dts) % C == 0:
            ckpt[len(dts)] = (x.clone(), t, cur)
    N = len(dts)
    x_final = x.clone()

    # dL/dx_N
    xr = device_to_real(grid, x_final).detach().requires_grad_(True)
    Lv = loss(xr)
    if not backward:
        return {"loss": float(Lv.detach()), "x_final": x_final, "steps": N}
    (g_xr,) = torch.autograd.grad(Lv, xr)
    lam = real_to_device(grid, g_xr.detach())

    g_sc = torch.zeros(grid.n, dtype=torch.float64, device=grid.device)
    g_B = torch.zeros(3, dtype=torch.float64, device=grid.device)
    g_k = torch.zeros((), dtype=torch.float64, device=grid.device)
    want_sc = material is not None
    iters = [0]

    def vjp(xs, v):
        return grid.vjp(xs, v, B, want_sc=want_sc)

    # the transposed step systems are solved on the device (one graph per
    # solve, FP64 context); a solve that reaches kmax without converging is
    # restarted on the host from its last iterate
    adj_grid = grid_for(params, idx, material, "fp64", kmax)

    seg_starts = sorted(k for k in ckpt if k < N) if N > 0 else []
    for s0 in reversed(seg_starts):
        s1 = min(s0 + C, N)
        xs = [ckpt[s0][0].clone()]
        t, cur = ckpt[s0][1], ckpt[s0][2]
        xw = xs[0].clone()
        for _ in range(s0, s1):
            t, cur = step(xw, t, cur)
            xs.append(xw.clone())
        for n in range(s1 - 1, s0 - 1, -1):
            h = 0.5 * dts[n]
            x_next, x_now = xs[n + 1 - s0], xs[n - s0]

            def matvec(v, x_next=x_next, h=h):
                iters[0] += 1
                return v - h * vjp(x_next, v)[0]

            mu, it, ok = adj_grid.adjoint_solve(x_next, lam, h, adjoint_tol, B)
            iters[0] += it
            if not ok:
                mu = _gmres(matvec, lam, adjoint_tol, x0=mu)
            gx1, gs1, _, gp1 = vjp(x_next, mu)
            gx0, gs0, _, gp0 = vjp(x_now, mu)
            lam = mu + h * gx0
            if want_sc:
                g_sc += h * (gs1 + gs0)
            g_B += h * (gp1[:3] + gp0[:3])
            g_k += h * (gp1[3] + gp0[3])

    return {
        "loss": float(Lv.detach()),
        "x_final": x_final,
        "grad_x0": device_to_real(grid, lam),
        "grad_sc": node_to_reference_order(grid, g_sc) if want_sc else None,
        "grad_B": g_B.cpu().numpy(),
        "grad_kappa": float(g_k),
        "steps": N,
        "adjoint_iters": iters[0],
    }


def box_mean_psi2(params, box: tuple) -> Callable[[torch.Tensor], torch.Tensor]:
    """Loss mean |psi|^2 over the interior nodes with i0 <= i < i1, j0 <= j < j1,
    k0 <= k < k1 (box = (i0, i1, j0, j1, k0, k1), full-grid indices), for the
    real layout (reference interior order: k fastest, then j, then i)."""
    Nx, Ny, Nz = int(params.Nx), int(params.Ny), int(params.Nz)
    nx, ny = Nx - 1, Ny - 1
    nz = Nz - 1 if Nz > 1 else 1
    ii, jj, kk = np.meshgrid(np.arange(1, Nx), np.arange(1, Ny), np.arange(1, Nz) if Nz > 1 else np.array([0]),
                             indexing="ij")
    i0, i1, j0, j1, k0, k1 = box
    sel = ((ii >= i0) & (ii < i1) & (jj >= j0) & (jj < j1) & (kk >= k0) & (kk < k1)).reshape(-1)
    idx = torch.as_tensor(np.nonzero(sel)[0])
    n = nx * ny * nz

    def loss(xr: torch.Tensor) -> torch.Tensor:
        j = idx.to(xr.device)
        return (xr[:n][j] ** 2 + xr[n:2 * n][j] ** 2).mean()

    return loss
