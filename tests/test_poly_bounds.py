"""The interval the polynomial preconditioner is built on: the spectrum of the
trapezoidal operator A = I - dt/2 J(x) lies in [1 - dt/2, 1 + dt/2 rho], rho
the Gershgorin bound the context computes from the stencil coefficients
(8 kappa^2 sum_a 1/h_a^2 + 6 for the vector-potential rows, (2 + 2 sqrt 2)
sum_a 1/h_a^2 + 4 (+ 1/tau with a material) for the order-parameter rows,
times 1.02).  J comes from the FP64 torch restatement of the RHS (oracle,
pinned to the reference's golden vectors) by forward-mode autodiff, and its
eigenvalues from a dense eigensolve.  Also the polynomial itself:
lambda p(lambda) stays within 1 +- 1 / T_{d+1}(theta / delta) on the interval
(the construction the device runs, restated here)."""

import numpy as np
import pytest
import torch

from oracle import tdgl_oracle as orc
from oracle import tdgl_torch_ref as tr

TAU = 0.1


def rho_bound(p, kappa2_max, has_material):
    s2 = 1 / p.hx ** 2 + 1 / p.hy ** 2 + (1 / p.hz ** 2 if p.Nz > 1 else 0.0)
    field = 8.0 * kappa2_max * s2 + 6.0
    order = (2.0 + 2.0 * np.sqrt(2.0)) * s2 + 4.0 + (1.0 / TAU if has_material else 0.0)
    return 1.02 * max(field, order)


def poly_coefficients(deg, dt, rho):
    """Horner coefficients in t = (lambda - theta) / delta, as the device builds them."""
    n = deg + 1
    h = dt / 2
    a, b = 1 - h, 1 + h * rho
    th, de = (a + b) / 2, (b - a) / 2
    x0 = th / de
    tm = np.zeros(n + 2); tm[0] = 1.0
    tc = np.zeros(n + 2); tc[1] = -1.0
    vm, vc = 1.0, x0
    for m in range(1, n):
        tn = np.zeros(n + 2)
        for k in range(m + 2):
            tn[k] = (-2.0 * tc[k - 1] if k > 0 else 0.0) - (tm[k] if k <= m - 1 else 0.0)
        tm, tc = tc, tn
        vm, vc = vc, 2 * x0 * vc - vm
    N = -tc[:n + 1] / vc
    N[0] += 1.0
    e = np.zeros(n)
    q = N[n]
    e[n - 1] = q / de
    for k in range(n - 1, 0, -1):
        q = N[k] + (-x0) * q
        e[k - 1] = q / de
    return e, th, de, a, b, vc


@pytest.mark.parametrize("deg", [1, 2, 3, 4, 8])
def test_polynomial_maps_interval_near_one(deg):
    e, th, de, a, b, tn = poly_coefficients(deg, 0.1, 384.0)
    lam = np.linspace(a, b, 4001)
    t = (lam - th) / de
    lp = lam * sum(e[k] * t ** k for k in range(deg + 1))
    assert np.max(np.abs(lp - 1.0)) <= 1.0 / tn * (1 + 1e-9)


def _operator(Nx, Ny, Nz, kappa, bz, dt, material=False, seed=0):
    import nanowire_tdgl_b200 as tb
    p = tb.SimulationParameters(Nx=Nx, Ny=Ny, Nz=Nz, hx=0.5, hy=0.5, hz=0.5, kappa=kappa)
    dev = tb.Device(p, applied_field=tb.AppliedField(Bz=bz, t_on_fraction=1.0))
    dev.add_hole([(2.0, 2.0), (4.0, 2.0), (4.0, 4.0), (2.0, 4.0)])
    g = orc.make_grid(dev.params, dev.idx, dev.material)
    X0 = dev.initial_state().data
    rng = np.random.default_rng(seed)
    n = p.n_interior
    X0[:n] = X0[:n] * (0.6 + 0.5 * rng.random(n)) * np.exp(1j * rng.standard_normal(n))
    x = torch.tensor(tr.to_real(X0, g))
    sc = None
    if material:
        sc = torch.tensor(np.where(rng.random(n) < 0.2, 0.0, 1.0))

    J = torch.func.jacfwd(lambda z: tr.eval_f(g, z, sc=sc, bz=bz))(x).numpy()
    return p, np.eye(x.numel()) - dt / 2 * J


@pytest.mark.parametrize("Nx,Ny,Nz,kappa,material", [(12, 10, 4, 2.0, False), (12, 10, 4, 4.0, True),
                                                      (14, 12, 1, 2.0, False)])
def test_spectrum_inside_interval(Nx, Ny, Nz, kappa, material):
    dt = 0.1
    p, A = _operator(Nx, Ny, Nz, kappa, 0.5, dt, material)
    lam = np.linalg.eigvals(A)
    rho = rho_bound(p, kappa ** 2, material)
    assert np.max(np.abs(lam)) <= 1 + dt / 2 * rho
    assert np.min(lam.real) >= 1 - dt / 2 - 1e-9
    # the top of the spectrum is real: the Chebyshev interval is the right shape
    top = lam[np.abs(lam) > 0.5 * np.max(np.abs(lam))]
    assert np.max(np.abs(top.imag)) < 1e-6 * np.max(np.abs(lam))
