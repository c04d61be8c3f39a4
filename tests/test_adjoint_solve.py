"""Device-resident adjoint solve (tdgl_adjoint_solve): the returned mu
satisfies (I - h J(x)^T) mu = b to the requested tolerance, checked with the
adjoint kernel itself; a solve capped by kmax reports it and returns an
iterate that a host restart completes."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(Nz, kmax=64, seed=3):
    import torch
    import nanowire_tdgl_b200 as tb
    from nanowire_tdgl_b200.engine import DeviceGrid
    p = tb.SimulationParameters(Nx=14, Ny=12, Nz=Nz, hx=0.5, hy=0.5, hz=0.5, kappa=2.5)
    dev = tb.Device(p, applied_field=tb.AppliedField(Bz=0.5, t_on_fraction=1.0))
    dev.add_hole([(2.0, 2.0), (3.5, 2.0), (3.5, 3.5), (2.0, 3.5)])
    rng = np.random.default_rng(seed)
    x0 = dev.initial_state()
    n = x0.psi.shape[0]
    x0.psi[:] += 0.1 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    x0.data[n:] = 0.05 * rng.standard_normal(x0.data.size - n)
    g = DeviceGrid(p, dev.idx, dev.material, "fp64", kmax, "gmres")
    x = g.pack(x0.data)
    bref = np.zeros(p.n_state, dtype=np.complex128)
    bref[:n] = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    bref[n:] = rng.standard_normal(p.n_state - n)
    b = g.pack(bref)
    torch.cuda.synchronize()
    return g, x, b


def _residual(g, x, b, mu, h, B):
    import torch
    amu = mu - h * g.vjp(x, mu, B, want_sc=False)[0]
    return float(torch.linalg.vector_norm(amu - b) / torch.linalg.vector_norm(b))


@pytest.mark.parametrize("Nz", [1, 6])
def test_device_adjoint_solve_residual(Nz):
    g, x, b = _setup(Nz)
    B = (0.0, 0.0, 0.5)
    mu, it, ok = g.adjoint_solve(x, b, 0.05, 1e-11, B)
    assert ok and 0 < it < 64
    assert _residual(g, x, b, mu, 0.05, B) < 1e-10


def test_device_adjoint_solve_capped_then_restarted():
    from nanowire_tdgl_b200.adjoint import _gmres
    g, x, b = _setup(6, kmax=4)
    B = (0.0, 0.0, 0.5)
    mu, it, ok = g.adjoint_solve(x, b, 0.05, 1e-11, B)
    assert not ok and it == 4
    r4 = _residual(g, x, b, mu, 0.05, B)
    assert r4 < 1.0                                    # the capped iterate already reduced the residual
    mu2 = _gmres(lambda v: v - 0.05 * g.vjp(x, v, B, want_sc=False)[0], b, 1e-11, x0=mu)
    assert _residual(g, x, b, mu2, 0.05, B) < 1e-10


def test_zero_right_hand_side():
    import torch
    g, x, b = _setup(6)
    mu, it, ok = g.adjoint_solve(x, torch.zeros_like(b), 0.05, 1e-11, (0.0, 0.0, 0.5))
    assert ok and it == 0 and not bool(torch.any(mu != 0))
