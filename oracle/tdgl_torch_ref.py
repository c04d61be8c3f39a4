"""Differentiable FP64 torch restatement of the TDGL right-hand side — TEST
INFRASTRUCTURE ONLY.

Used by ``tests/`` as the independent reference for the hand-written adjoint
(vector-Jacobian product) kernels and for the gradients of the trapezoidal
stepper: torch autograd through this file gives d(v . f)/d(x, s, Bz, kappa)
without any of the product code.  The product package never imports it.

It follows ``oracle/tdgl_oracle.py`` (which is pinned against the reference's
golden vectors) line for line, in real arithmetic:
  boundary procedure   src/tdgl3d/physics/rhs.py:54-139
  RHS assembly         src/tdgl3d/physics/rhs.py:147-239
  operators            src/tdgl3d/operators/sparse_operators.py:35-317

State layout (``real`` layout): a real tensor of length ncomp * n, blocks
[psi_re, psi_im, phi_x, phi_y, (phi_z)], interior nodes in the reference's
order (``GridIndices.interior_to_full``, k fastest).  Parameters: the interior
superconducting mask sc (``MaterialMap.interior_sc_mask`` = 1 - s for a
suppression field s; None for no material), the applied field (bx, by, bz) and
a uniform kappa — each a float or a 0-d tensor that may require gradients.
"""

from __future__ import annotations

import numpy as np
import torch

from .tdgl_oracle import TAU_RELAX, OracleGrid


def _full(g: OracleGrid, v: torch.Tensor) -> torch.Tensor:
    nx, ny = g.Nx - 1, g.Ny - 1
    nz = g.Nz - 1 if g.is_3d else 1
    out = torch.zeros(g.shape, dtype=v.dtype, device=v.device)
    out[g.int_sel] = v.reshape(nx, ny, nz).permute(2, 1, 0)
    return out


def _back(a: torch.Tensor) -> torch.Tensor:
    return a.permute(2, 1, 0).reshape(-1)


def _sh(a: torch.Tensor, dk: int, dj: int, di: int) -> torch.Tensor:
    nk, nj, ni = a.shape
    ks = slice(1 + dk, nk - 1 + dk) if nk > 1 else slice(0, 1)
    return a[ks, 1 + dj:nj - 1 + dj, 1 + di:ni - 1 + di]


def boundary_fields(g: OracleGrid, x: torch.Tensor, bx, by, bz):
    """Full-grid (psi_re, psi_im, phi_x, phi_y, phi_z) after the reference's
    boundary procedure (same steps as tdgl_oracle.boundary_fields)."""
    n = g.n
    pr, pi = _full(g, x[:n]), _full(g, x[n:2 * n])
    fx, fy = _full(g, x[2 * n:3 * n]), _full(g, x[3 * n:4 * n])
    fz = _full(g, x[4 * n:5 * n]) if g.is_3d else torch.zeros_like(pr)
    Nx, Ny, Nz = g.Nx, g.Ny, g.Nz
    fx = fx.clone()
    fx[:, :, [0, Nx - 1]] = 0.0
    fy = fy.clone()
    fy[:, [0, Ny - 1], :] = 0.0
    if g.is_3d:
        fz = fz.clone()
        fz[[0, Nz - 1], :, :] = 0.0
    r0, i0, x0, y0, z0 = pr, pi, fx, fy, fz
    pr, pi, fx, fy, fz = pr.clone(), pi.clone(), fx.clone(), fy.clone(), fz.clone()
    czxy = bz * g.hx * g.hy
    cyzx = by * g.hz * g.hx
    cxyz = bx * g.hy * g.hz
    kk = slice(1, Nz) if g.is_3d else slice(0, 1)
    jj, ii = slice(1, Ny), slice(1, Nx)

    def rot(re, im, ang):        # (re + i im) e^{i ang}
        c, s = torch.cos(ang), torch.sin(ang)
        return re * c - im * s, re * s + im * c

    if g.periodic[0]:
        pr[kk, jj, 0] = r0[kk, jj, Nx - 1]; pi[kk, jj, 0] = i0[kk, jj, Nx - 1]
        pr[kk, jj, Nx] = r0[kk, jj, 1]; pi[kk, jj, Nx] = i0[kk, jj, 1]
        fx[kk, jj, 0] = x0[kk, jj, Nx - 1]
        fx[kk, jj, Nx] = x0[kk, jj, 1]
    else:
        a, b = rot(r0[kk, jj, 1], i0[kk, jj, 1], -x0[kk, jj, 0])
        pr[kk, jj, 0] = a; pi[kk, jj, 0] = b
        a, b = rot(r0[kk, jj, Nx - 1], i0[kk, jj, Nx - 1], x0[kk, jj, Nx - 1])
        pr[kk, jj, Nx] = a; pi[kk, jj, Nx] = b
        fy[kk, jj, 0] = -czxy + y0[kk, jj, 1]
        fy[kk, jj, Nx] = czxy + y0[kk, jj, Nx - 1]
        fz[kk, jj, 0] = cyzx + z0[kk, jj, 1]
        fz[kk, jj, Nx] = -cyzx + z0[kk, jj, Nx - 1]
    if g.periodic[1]:
        pr[kk, 0, ii] = r0[kk, Ny - 1, ii]; pi[kk, 0, ii] = i0[kk, Ny - 1, ii]
        pr[kk, Ny, ii] = r0[kk, 1, ii]; pi[kk, Ny, ii] = i0[kk, 1, ii]
        fy[kk, 0, ii] = y0[kk, Ny - 1, ii]
        fy[kk, Ny, ii] = y0[kk, 1, ii]
    else:
        a, b = rot(r0[kk, 1, ii], i0[kk, 1, ii], -y0[kk, 0, ii])
        pr[kk, 0, ii] = a; pi[kk, 0, ii] = b
        a, b = rot(r0[kk, Ny - 1, ii], i0[kk, Ny - 1, ii], y0[kk, Ny - 1, ii])
        pr[kk, Ny, ii] = a; pi[kk, Ny, ii] = b
        fx[kk, 0, ii] = czxy + x0[kk, 1, ii]
        fx[kk, Ny, ii] = -czxy + x0[kk, Ny - 1, ii]
        fz[kk, 0, ii] = -cxyz + z0[kk, 1, ii]
        fz[kk, Ny, ii] = cxyz + z0[kk, Ny - 1, ii]
    if g.is_3d:
        if g.periodic[2]:
            pr[0, jj, ii] = r0[Nz - 1, jj, ii]; pi[0, jj, ii] = i0[Nz - 1, jj, ii]
            pr[Nz, jj, ii] = r0[1, jj, ii]; pi[Nz, jj, ii] = i0[1, jj, ii]
            fz[0, jj, ii] = z0[Nz - 1, jj, ii]
            fz[Nz, jj, ii] = z0[1, jj, ii]
        else:
            a, b = rot(r0[1, jj, ii], i0[1, jj, ii], -z0[0, jj, ii])
            pr[0, jj, ii] = a; pi[0, jj, ii] = b
            a, b = rot(r0[Nz - 1, jj, ii], i0[Nz - 1, jj, ii], z0[Nz - 1, jj, ii])
            pr[Nz, jj, ii] = a; pi[Nz, jj, ii] = b
            fx[0, jj, ii] = -cyzx + x0[1, jj, ii]
            fx[Nz, jj, ii] = cyzx + x0[Nz - 1, jj, ii]
            fy[0, jj, ii] = cxyz + y0[1, jj, ii]
            fy[Nz, jj, ii] = -cxyz + y0[Nz - 1, jj, ii]
    dev = x.device
    fx = fx * (~torch.as_tensor(g.hole[0], device=dev))
    fy = fy * (~torch.as_tensor(g.hole[1], device=dev))
    if g.is_3d:
        fz = fz * (~torch.as_tensor(g.hole[2], device=dev))
    return pr, pi, fx, fy, fz


def eval_f(g: OracleGrid, x: torch.Tensor, sc=None, bx=0.0, by=0.0, bz=0.0, kappa=None) -> torch.Tensor:
    """dX/dt in the real layout (see the module docstring); same sums as
    tdgl_oracle.eval_f.  ``sc``: interior sc mask (reference order) or None;
    ``kappa``: uniform kappa (defaults to the grid's), ignored where the grid
    carries per-node kappa."""
    pr, pi, fx, fy, fz = boundary_fields(g, x, bx, by, bz)
    d3 = g.is_3d
    hx, hy, hz = g.hx, g.hy, g.hz
    cr, ci = _sh(pr, 0, 0, 0), _sh(pi, 0, 0, 0)

    def lap_psi(f, off_m, off_p, ang_m, ang_p):
        # e^{-i ang_m} psi(m - d) - 2 psi(m) + e^{i ang_p} psi(m + d)
        mr, mi = _sh(pr, *off_m), _sh(pi, *off_m)
        pr_, pi_ = _sh(pr, *off_p), _sh(pi, *off_p)
        cm, sm = torch.cos(ang_m), torch.sin(ang_m)
        cp, sp = torch.cos(ang_p), torch.sin(ang_p)
        re = (cm * mr + sm * mi) - 2.0 * cr + (cp * pr_ - sp * pi_)
        im = (cm * mi - sm * mr) - 2.0 * ci + (cp * pi_ + sp * pr_)
        return re, im

    lxr, lxi = lap_psi(fx, (0, 0, -1), (0, 0, 1), _sh(fx, 0, 0, -1), _sh(fx, 0, 0, 0))
    lyr, lyi = lap_psi(fy, (0, -1, 0), (0, 1, 0), _sh(fy, 0, -1, 0), _sh(fy, 0, 0, 0))
    dr = lxr / hx ** 2 + lyr / hy ** 2
    di = lxi / hx ** 2 + lyi / hy ** 2
    if d3:
        lzr, lzi = lap_psi(fz, (-1, 0, 0), (1, 0, 0), _sh(fz, -1, 0, 0), _sh(fz, 0, 0, 0))
        dr = dr + lzr / hz ** 2
        di = di + lzi / hz ** 2
    m2 = cr * cr + ci * ci
    glr, gli = (1.0 - m2) * cr, (1.0 - m2) * ci
    if sc is not None:
        s = _full(g, sc)[g.int_sel]
        dr = dr + s * glr - (1.0 - s) * cr / TAU_RELAX
        di = di + s * gli - (1.0 - s) * ci / TAU_RELAX
    else:
        dr = dr + glr
        di = di + gli

    if g.kappa_int is not None:
        k2 = _full(g, torch.as_tensor(g.kappa_int, dtype=x.dtype, device=x.device))[g.int_sel] ** 2
    else:
        kap = g.kappa if kappa is None else kappa
        k2 = kap * kap * torch.ones_like(cr)
    cx, cy = k2 / hx ** 2, k2 / hy ** 2
    cz = k2 / hz ** 2 if d3 else torch.zeros_like(k2)

    def lap(f, wx, wy, wz):
        out = (-2.0 * (wx + wy + wz)) * _sh(f, 0, 0, 0)
        out = out + wx * (_sh(f, 0, 0, -1) + _sh(f, 0, 0, 1)) + wy * (_sh(f, 0, -1, 0) + _sh(f, 0, 1, 0))
        if d3:
            out = out + wz * (_sh(f, -1, 0, 0) + _sh(f, 1, 0, 0))
        return out

    def sup(f, dk, dj, dii):
        # Im[e^{-i f(m)} conj(psi(m)) psi(m + a)]
        a0 = _sh(f, 0, 0, 0)
        c0, s0 = torch.cos(a0), torch.sin(a0)
        ur, ui = c0 * cr - s0 * ci, -(s0 * cr + c0 * ci)
        return ur * _sh(pi, dk, dj, dii) + ui * _sh(pr, dk, dj, dii)

    def curl(fb, wb, a, b):
        ak, aj, ai = a
        bk, bj, bi = b
        return wb * (-_sh(fb, ak, aj, ai) + _sh(fb, 0, 0, 0) + _sh(fb, ak - bk, aj - bj, ai - bi) - _sh(fb, -bk, -bj, -bi))

    ex, ey, ez = (0, 0, 1), (0, 1, 0), (1, 0, 0)
    dfx = lap(fx, 2 * cx, cy, cz) + sup(fx, *ex) + curl(fy, cy, ex, ey)
    dfy = lap(fy, cx, 2 * cy, cz) + sup(fy, *ey) + curl(fx, cx, ey, ex)
    outs = [_back(dr), _back(di)]
    hole = [torch.as_tensor(h, device=x.device) for h in g.hole_int]
    if d3:
        dfx = dfx + curl(fz, cz, ex, ez)
        dfy = dfy + curl(fz, cz, ey, ez)
        dfz = lap(fz, cx, cy, 2 * cz) + sup(fz, *ez) + curl(fx, cx, ez, ex) + curl(fy, cy, ez, ey)
    outs.append(_back(dfx) * (~hole[0]))
    outs.append(_back(dfy) * (~hole[1]))
    if d3:
        outs.append(_back(dfz) * (~hole[2]))
    return torch.cat(outs)


def to_real(X: np.ndarray, g: OracleGrid) -> np.ndarray:
    """Reference complex128 state -> real layout (link imaginary parts dropped)."""
    n = g.n
    parts = [X[:n].real, X[:n].imag, X[n:2 * n].real, X[2 * n:3 * n].real]
    if g.is_3d:
        parts.append(X[3 * n:4 * n].real)
    return np.concatenate(parts)


def from_real(x: np.ndarray, g: OracleGrid) -> np.ndarray:
    """Real layout -> reference complex128 state."""
    n = g.n
    nc = 5 if g.is_3d else 4
    out = [x[:n] + 1j * x[n:2 * n]] + [x[c * n:(c + 1) * n].astype(np.complex128) for c in range(2, nc)]
    return np.concatenate(out)
