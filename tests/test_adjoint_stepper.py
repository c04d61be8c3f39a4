"""Gradients through the trapezoidal stepper (differentiation form) against
central finite differences of the device stepper and against an FP64 torch
reference gradient (states from exact-Newton trapezoidal steps and Jacobians
by torch autograd of the torch restatement, dense transposed solves).

Tolerances: finite differences (eps 1e-5 on a tight-tolerance FP64 forward)
agree to 1e-4 relative (the target of the differentiation form); the torch
reference agrees to 1e-7 relative.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

B = (0.0, 0.0, 0.4)
T_STOP, DT = 0.6, 0.1
TOL = dict(newton_tol_f=1e-13, newton_tol_dx=1e-11, tol_gcr=1e-13, newton_max_iter=30, kmax=128)
BOX = (2, 6, 2, 5, 1, 3)


def _setup(kappa=2.0, sc_shift=None):
    import nanowire_tdgl_b200 as tb
    p = tb.SimulationParameters(Nx=8, Ny=7, Nz=4, hx=0.5, hy=0.5, hz=0.5, kappa=kappa)
    idx = tb.construct_indices(p)
    rng = np.random.default_rng(11)
    s_full = 0.3 * rng.random(p.dim_x)                   # suppression field s(x)
    sc_full = 1.0 - s_full
    mat = tb.MaterialMap(kappa=np.full(p.dim_x, kappa), sc_mask=sc_full.copy(),
                         interior_sc_mask=sc_full[np.asarray(idx.interior_to_full)].copy())
    if sc_shift is not None:
        r, e = sc_shift
        mat.interior_sc_mask[r] += e
    n = p.n_interior
    x0 = np.zeros(p.n_state, dtype=np.complex128)
    x0[:n] = 1.0 + 0.05 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    x0[n:] = 0.02 * rng.standard_normal(p.n_state - n)
    return p, idx, mat, x0


def _run(p, idx, mat, x0, Bv=B, backward=True, ckpt=4):
    import nanowire_tdgl_b200 as tb
    return tb.trapezoidal_gradient(x0, p, idx, 0.0, T_STOP, DT, tb.box_mean_psi2(p, BOX), material=mat, B=Bv,
                                   checkpoint_every=ckpt, precision="fp64", backward=backward, **TOL)


def _close(a, b, rel):
    return abs(a - b) <= rel * max(abs(b), 1e-8)


def test_gradient_matches_finite_differences():
    p, idx, mat, x0 = _setup()
    res = _run(p, idx, mat, x0)
    assert res["steps"] == 6
    eps = 1e-5
    # field
    lp = _run(p, idx, mat, x0, (0.0, 0.0, B[2] + eps), backward=False)["loss"]
    lm = _run(p, idx, mat, x0, (0.0, 0.0, B[2] - eps), backward=False)["loss"]
    assert _close(res["grad_B"][2], (lp - lm) / (2 * eps), 1e-4), (res["grad_B"][2], (lp - lm) / (2 * eps))
    # kappa (uniform, through the material map)
    lp = _run(*(_setup(kappa=2.0 + eps)[:3]), x0, backward=False)["loss"]
    lm = _run(*(_setup(kappa=2.0 - eps)[:3]), x0, backward=False)["loss"]
    assert _close(res["grad_kappa"], (lp - lm) / (2 * eps), 1e-4), (res["grad_kappa"], (lp - lm) / (2 * eps))
    # superconducting mask at a few interior nodes (reference order)
    gsc = res["grad_sc"].cpu().numpy()
    for r in (7, 40, 77):
        lp = _run(*(_setup(sc_shift=(r, eps))[:3]), x0, backward=False)["loss"]
        lm = _run(*(_setup(sc_shift=(r, -eps))[:3]), x0, backward=False)["loss"]
        assert _close(gsc[r], (lp - lm) / (2 * eps), 1e-4), (r, gsc[r], (lp - lm) / (2 * eps))
    # initial state: psi_re, psi_im, phi_x entries (real layout)
    g0 = res["grad_x0"].cpu().numpy()
    n = p.n_interior
    for q in (12, n + 30, 2 * n + 55):
        xp, xm = x0.copy(), x0.copy()
        comp = 1j if n <= q < 2 * n else 1.0
        k = q - n if n <= q < 2 * n else (q if q < n else q - n)
        xp[k] += eps * comp
        xm[k] -= eps * comp
        lp = _run(p, idx, mat, xp, backward=False)["loss"]
        lm = _run(p, idx, mat, xm, backward=False)["loss"]
        assert _close(g0[q], (lp - lm) / (2 * eps), 1e-4), (q, g0[q], (lp - lm) / (2 * eps))


def test_checkpointing_does_not_change_the_gradient():
    p, idx, mat, x0 = _setup()
    a = _run(p, idx, mat, x0, ckpt=1)
    b = _run(p, idx, mat, x0, ckpt=50)
    assert np.allclose(a["grad_x0"].cpu().numpy(), b["grad_x0"].cpu().numpy(), rtol=0, atol=1e-12)
    assert abs(a["grad_B"][2] - b["grad_B"][2]) < 1e-12


def test_gradient_matches_torch_double_reference():
    from oracle import tdgl_oracle as orc
    from oracle import tdgl_torch_ref as tr
    p, idx, mat, x0 = _setup()
    res = _run(p, idx, mat, x0)
    g = orc.make_grid(p, idx, mat)
    import dataclasses
    g = dataclasses.replace(g, kappa_int=None, kappa=2.0)   # the material's kappa is uniform: make it a parameter
    sc0 = torch.tensor(g.sc_int)

    def f0(x):
        return tr.eval_f(g, x, sc0, 0.0, 0.0, B[2], kappa=2.0)

    # forward states: trapezoidal steps with exact (dense-Jacobian) Newton in FP64 torch
    xs = [torch.tensor(tr.to_real(x0, g))]
    times = [0.0]
    t = 0.0
    while t < T_STOP - 1e-14:
        h = min(DT, T_STOP - t)
        xn = xs[-1]
        fn = f0(xn)
        gam = xn + 0.5 * h * fn
        x = xn + h * fn
        for _ in range(30):
            gv = x - 0.5 * h * f0(x) - gam
            if float(gv.abs().max()) < 1e-14:
                break
            J = torch.autograd.functional.jacobian(f0, x)
            x = x + torch.linalg.solve(torch.eye(J.shape[0], dtype=torch.float64) - 0.5 * h * J, -gv)
        xs.append(x)
        t += h
        times.append(t)
    sc = torch.tensor(g.sc_int)
    kap = torch.tensor(2.0, dtype=torch.float64)
    bz = torch.tensor(B[2], dtype=torch.float64)

    def f(x, sc_=sc, kap_=kap, bz_=bz):
        return tr.eval_f(g, x, sc_, 0.0, 0.0, bz_, kappa=kap_)

    loss = __import__("nanowire_tdgl_b200").box_mean_psi2(p, BOX)
    xN = xs[-1].clone().requires_grad_(True)
    (lam,) = torch.autograd.grad(loss(xN), xN)
    g_sc = torch.zeros_like(sc)
    g_k = 0.0
    g_b = 0.0
    for n in range(len(xs) - 2, -1, -1):
        h = 0.5 * (times[n + 1] - times[n])
        J1 = torch.autograd.functional.jacobian(f, xs[n + 1])
        A = torch.eye(J1.shape[0], dtype=torch.float64) - h * J1
        mu = torch.linalg.solve(A.T, lam)
        for xx in (xs[n + 1], xs[n]):
            xv = xx.clone().requires_grad_(True)
            sc_v = sc.clone().requires_grad_(True)
            kv = kap.clone().requires_grad_(True)
            bv = bz.clone().requires_grad_(True)
            val = (mu * f(xv, sc_v, kv, bv)).sum()
            gx, gs, gk, gb = torch.autograd.grad(val, (xv, sc_v, kv, bv))
            g_sc += h * gs
            g_k += h * float(gk)
            g_b += h * float(gb)
            if xx is xs[n]:
                lam = mu + h * gx
    ref_x0 = lam.numpy()
    got = res["grad_x0"].cpu().numpy()
    assert np.max(np.abs(got - ref_x0)) <= 1e-7 * np.max(np.abs(ref_x0))
    assert np.max(np.abs(res["grad_sc"].cpu().numpy() - g_sc.numpy())) <= 1e-7 * np.max(np.abs(g_sc.numpy()))
    assert _close(res["grad_kappa"], g_k, 1e-7)
    assert _close(res["grad_B"][2], g_b, 1e-7)
