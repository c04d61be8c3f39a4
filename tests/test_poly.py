"""Polynomial (Chebyshev) right preconditioner of the analytic-product GMRES
solves: every degree reproduces the reference's trapezoidal trajectory
(against the oracle, which runs the reference's unpreconditioned
finite-difference GCR), the Krylov iterations fall as the degree grows, and
the setting is validated."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

T_STOP = 0.5
KW = dict(newton_tol_f=1e-8, newton_tol_dx=1e-3, tol_gcr=1e-6)


@pytest.fixture(scope="module")
def tb():
    import nanowire_tdgl_b200 as tb
    return tb


def _case(tb, kappa=2.0, periodic_x=False):
    p = tb.SimulationParameters(Nx=14, Ny=10, Nz=4, hx=0.5, hy=0.5, hz=0.5, kappa=kappa, periodic_x=periodic_x)
    dev = tb.Device(p, applied_field=tb.AppliedField(Bz=0.5, t_on_fraction=1.0))
    dev.add_hole([(3.0, 2.0), (5.0, 2.0), (5.0, 4.0), (3.0, 4.0)])
    x0 = dev.initial_state()
    rng = np.random.default_rng(3)
    n = x0.psi.shape[0]
    x0.psi += 0.02 * (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * dev.material.interior_sc_mask
    return dev, x0.data


def _grid(dev, precision):
    from nanowire_tdgl_b200.engine import grid_for
    from nanowire_tdgl_b200.solvers import DEFAULT_KMAX
    return grid_for(dev.params, dev.idx, dev.material, precision, DEFAULT_KMAX, "gmres")


def _run(tb, dev, x0, precision, degree):
    g = _grid(dev, precision)
    g.set_poly(degree)
    try:
        st = {}
        fs = tb.FieldSchedule(dev.applied_field, dev.params, dev.idx, T_STOP)
        times, hist = tb.trapezoidal(x0, dev.params, dev.idx, fs, 0.0, T_STOP, 0.1, progress=False,
                                     material=dev.material, precision=precision, jvp="analytic", stats=st, **KW)
    finally:
        g.set_poly(-1)
    return np.asarray(times), np.asarray(hist), st


def _oracle(dev, x0):
    from oracle import tdgl_oracle as orc
    g = orc.make_grid(dev.params, dev.idx, dev.material)
    fld = orc.field_schedule(Bz=0.5, t_on_fraction=1.0, t_stop=T_STOP)
    return orc.trapezoidal(x0, g, fld, 0.0, T_STOP, 0.1, **KW)


@pytest.mark.parametrize("periodic_x", [False, True])
def test_every_degree_matches_oracle_fp64(tb, periodic_x):
    dev, x0 = _case(tb, periodic_x=periodic_x)
    times_ref, hist_ref = _oracle(dev, x0)
    iters = {}
    for degree in (0, 1, 3, 8):
        times, hist, st = _run(tb, dev, x0, "fp64", degree)
        assert np.allclose(times, times_ref, rtol=0, atol=1e-14), degree
        # Newton converges to tol_f 1e-8 whichever linear solver it uses
        assert np.max(np.abs(hist - hist_ref)) < 1e-7, degree
        iters[degree] = st["krylov_iters"]
    assert iters[3] < iters[0] and iters[8] <= iters[3], iters


@pytest.mark.parametrize("kappa", [2.0, 4.0])
def test_mixed_degrees_track_fp64(tb, kappa):
    dev, x0 = _case(tb, kappa=kappa)
    _, ref, _ = _run(tb, dev, x0, "fp64", 0)
    n = dev.params.n_interior
    p_ref = np.abs(ref[:n, -1]) ** 2
    for degree in (0, 2, 3, 6):
        _, mix, st = _run(tb, dev, x0, "mixed", degree)
        p_mix = np.abs(mix[:n, -1]) ** 2
        assert np.linalg.norm(p_mix - p_ref) / np.linalg.norm(p_ref) < 1e-6, (kappa, degree)
        assert st["krylov_iters"] > 0


def test_poly_setting_is_validated(tb):
    from nanowire_tdgl_b200._lib import TDGLError
    dev, _ = _case(tb)
    g = _grid(dev, "mixed")
    for bad in (-2, 13):
        with pytest.raises(TDGLError):
            g.set_poly(bad)
    g.set_poly(5)
    assert g.poly_degree == 5
    g.set_poly(0)
    assert g.poly_degree == 0
    g.set_poly(-1)
    assert 0 <= g.poly_degree <= 12
