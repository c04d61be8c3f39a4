"""Parity of the CUDA path (through the C ABI) with the reference's golden
vectors and with the oracle.  Tolerances:

* RHS, pack/unpack, observables: FP64, 1e-12 relative (summation order only);
  the layout permutation is bit-exact.
* TGCR / Newton: the reference's finite-difference product; GCR with CGS
  instead of MGS (identical in exact arithmetic): 1e-6 relative on the
  solution, identical iteration counts and convergence flags.
* Trajectories: Newton tolerance level, 1e-7 absolute on the state.
"""

import numpy as np
import pytest
import torch

from conftest import device_from_fixture, golden, golden_names

pytestmark = pytest.mark.gpu

CASES = golden_names("case_")
TRAPS = [n for n in golden_names("trap_") if n != "trap_config1"]


@pytest.fixture(scope="module")
def tb():
    import nanowire_tdgl_b200 as tb
    assert torch.cuda.is_available()
    return tb


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("name", CASES)
def test_eval_f_matches_reference(tb, name):
    d = golden(name)
    dev = device_from_fixture(d)
    u = tb.BoundaryVectors(d["u_Bx"], d["u_By"], d["u_Bz"])
    F = tb.eval_f(d["X_seeded"], dev.params, dev.idx, u, material=dev.material)
    assert _rel(F, d["F_seeded"]) < 1e-12
    if "X_random" in d:
        F = tb.eval_f(d["X_random"], dev.params, dev.idx, u, material=dev.material)
        assert _rel(F, d["F_random"]) < 1e-12


@pytest.mark.parametrize("name", ["case_3d_hole_edge", "case_2d_hole_triangle", "case_config1"])
def test_pack_unpack_bit_exact(tb, name):
    from nanowire_tdgl_b200.engine import grid_for
    d = golden(name)
    dev = device_from_fixture(d)
    g = grid_for(dev.params, dev.idx, dev.material)
    X = d["X_seeded"]
    back = g.unpack(g.pack(X)).cpu().numpy()
    assert np.array_equal(back, X)


@pytest.mark.parametrize("name", ["case_3d_basic", "case_3d_hole", "case_trilayer", "case_2d_basic"])
def test_jvp_matches_central_difference(tb, name):
    from nanowire_tdgl_b200.engine import grid_for
    from oracle import tdgl_oracle as orc
    d = golden(name)
    dev = device_from_fixture(d)
    og = orc.make_grid(dev.params, dev.idx, dev.material)
    g = grid_for(dev.params, dev.idx, dev.material)
    X = d.get("X_random", d["X_seeded"])
    rng = np.random.default_rng(2)
    P = rng.standard_normal(dev.params.n_state) + 0j
    dt, h = 0.1, 1e-5
    fd = (orc.eval_f(X + h * P, og, *d["B"]) - orc.eval_f(X - h * P, og, *d["B"])) / (2 * h)
    want = P - dt / 2 * fd
    ap = g.unpack(g.jvp(g.pack(X), g.pack(P), dt, "analytic", B=d["B"])).cpu().numpy()
    assert _rel(ap, want) < 1e-8
    ap_fd = g.unpack(g.jvp(g.pack(X), g.pack(P), dt, "fd", 1e-4, B=d["B"])).cpu().numpy()
    assert _rel(ap_fd, want) < 1e-3


@pytest.mark.parametrize("krylov", ["gcr", "gmres"])
@pytest.mark.parametrize("name", ["solver_3d_basic", "solver_3d_hole", "solver_2d_basic"])
def test_tgcr_and_newton_match_reference(tb, name, krylov):
    d = golden(name)
    case = golden("case_" + name[len("solver_"):])
    dev = device_from_fixture(case)
    f = tb.make_eval_f(dev.params, dev.idx, tuple(case["B"]), dev.material, krylov=krylov)
    dt = float(d["dt"])
    x = tb.tgcr_matrix_free_trap(f, d["x_lin"], d["b"], dt, tol=float(d["tgcr_tol"]))
    # GCR applies the finite-difference product along the reference's own
    # directions (agreement to rounding); GMRES along the normalised Arnoldi
    # vectors, so the O(eps_mf) truncation of the product differs at ~1e-5
    assert x.size and _rel(x, d["tgcr_x"]) < (1e-6 if krylov == "gcr" else 1e-4)
    xn, ok, it = tb.newton_gcr_trap(f, d["x_pred"], d["gamma"], dt, tol_f=1e-8, tol_dx=1e-3, max_iter=20,
                                    tol_gcr=1e-6)
    assert ok == bool(d["newton_converged"]) and it == int(d["newton_iters"])
    assert np.max(np.abs(xn - d["newton_x"])) < 1e-8


def test_tgcr_edge_cases(tb):
    d = golden("case_3d_basic")
    dev = device_from_fixture(d)
    f = tb.make_eval_f(dev.params, dev.idx, (0.0, 0.0, 0.0), dev.material)
    X = d["X_seeded"]
    b = 0.01 * d["X_random"]
    assert tb.tgcr_matrix_free_trap(f, X, b, 0.1, max_iter=0).size == 0           # no iteration allowed
    z = tb.tgcr_matrix_free_trap(f, X, np.zeros_like(b), 0.1)                        # b == 0
    assert z.size == b.size and not np.any(z)
    ident = tb.tgcr_matrix_free_trap(f, X, b, 0.0, tol=1e-8)                         # dt = 0: identity
    assert np.max(np.abs(ident - b)) < 1e-12 * np.max(np.abs(b)) + 1e-18


@pytest.mark.parametrize("name", TRAPS)
@pytest.mark.parametrize("jvp,krylov", [("fd", "gcr"), ("fd", "gmres"), ("analytic", "gmres")])
def test_trapezoidal_matches_reference(tb, name, jvp, krylov):
    d = golden(name)
    case = golden("case_" + name[len("trap_"):])
    dev = device_from_fixture(case)
    sol = tb.solve(dev, t_start=0.0, t_stop=float(d["t_stop"]), dt=float(d["dt"]), method="trapezoidal",
                   x0=d["x0"], progress=False, log_metadata=False, newton_tol_f=1e-8, newton_tol_dx=1e-3,
                   tol_gcr=1e-6, jvp=jvp, krylov=krylov)
    assert np.array_equal(sol.times, d["times"])
    err = np.max(np.abs(sol.states[:, d["saved_steps"]] - d["states"]))
    assert err < 1e-7, err


@pytest.mark.parametrize("krylov", ["gcr", "gmres"])
def test_trapezoidal_config1_101_steps(tb, krylov):
    d = golden("trap_config1")
    case = golden("case_config1")
    dev = device_from_fixture(case)
    sol = tb.solve(dev, t_start=0.0, t_stop=float(d["t_stop"]), dt=float(d["dt"]), method="trapezoidal",
                   x0=d["x0"], progress=False, log_metadata=False, newton_tol_f=1e-8, newton_tol_dx=1e-3,
                   tol_gcr=1e-6, krylov=krylov)
    assert len(sol.times) == 102 and np.array_equal(sol.times, d["times"])
    err = np.max(np.abs(sol.states[:, d["saved_steps"]] - d["states"]))
    assert err < 1e-7, err
    # observables of the final state, as the reference's Solution computes them
    assert np.allclose(sol.psi_squared(-1), d["psi2"], rtol=0, atol=1e-7)
    for mine, ref in zip(sol.bfield(-1), (d["Bx"], d["By"], d["Bz"])):
        assert np.allclose(mine, ref, rtol=0, atol=1e-6)
    for mine, ref in zip(sol.supercurrent_density(-1), (d["Jx"], d["Jy"], d["Jz"])):
        assert np.allclose(mine, ref, rtol=0, atol=1e-7)


@pytest.mark.parametrize("name", TRAPS)
def test_observables_match_reference(tb, name):
    d = golden(name)
    case = golden("case_" + name[len("trap_"):])
    dev = device_from_fixture(case)
    sol = tb.Solution(times=d["times"], states=d["states"], params=dev.params, idx=dev.idx, device=dev)
    assert np.allclose(sol.psi_squared(-1), d["psi2"], rtol=0, atol=1e-14)
    for mine, ref in zip(sol.bfield(-1), (d["Bx"], d["By"], d["Bz"])):
        assert np.allclose(mine, ref, rtol=0, atol=1e-12)
    for mine, ref in zip(sol.supercurrent_density(-1), (d["Jx"], d["Jy"], d["Jz"])):
        assert np.allclose(mine, ref, rtol=0, atol=1e-13)


def test_forward_euler_matches_reference(tb):
    d = golden("euler_3d_hole")
    case = golden("case_3d_hole")
    dev = device_from_fixture(case)
    sol = tb.solve(dev, t_start=0.0, t_stop=float(d["t_stop"]), dt=float(d["dt"]), method="euler",
                   x0=d["x0"], progress=False, log_metadata=False)
    assert np.allclose(sol.times, d["times"], rtol=0, atol=1e-15)
    assert _rel(sol.states[:, d["saved_steps"]], d["states"]) < 1e-11


def test_mixed_precision_against_fp64(tb):
    d = golden("trap_config1")
    case = golden("case_config1")
    dev = device_from_fixture(case)
    kw = dict(t_start=0.0, t_stop=2.0, dt=0.1, method="trapezoidal", x0=d["x0"], progress=False,
              log_metadata=False, newton_tol_f=1e-8, newton_tol_dx=1e-3, tol_gcr=1e-6, save_every=20)
    ref = tb.solve(dev, precision="fp64", **kw)
    mix = tb.solve(dev, precision="mixed", **kw)
    p_ref = np.abs(ref.psi(-1)) ** 2
    p_mix = np.abs(mix.psi(-1)) ** 2
    assert np.linalg.norm(p_mix - p_ref) / np.linalg.norm(p_ref) < 1e-6


def test_dt_min_and_nonconvergence_errors(tb):
    d = golden("case_3d_basic")
    dev = device_from_fixture(d)
    with pytest.raises(RuntimeError, match="dt reduced below dt_min"):
        tb.trapezoidal(d["X_seeded"], dev.params, dev.idx, tb.FieldSchedule(dev.applied_field, dev.params,
                       dev.idx, 1.0), 0.0, 1.0, 0.1, newton_max_iter=0, dt_min=0.05, progress=False)
    with pytest.raises(RuntimeError, match="Newton did not converge"):
        tb.trapezoidal(d["X_seeded"], dev.params, dev.idx, tb.FieldSchedule(dev.applied_field, dev.params,
                       dev.idx, 1.0), 0.0, 1.0, 0.1, newton_max_iter=0, adaptive=False, progress=False)


def test_nonfinite_state_is_reported(tb):
    from nanowire_tdgl_b200._lib import TDGLError
    d = golden("case_3d_basic")
    dev = device_from_fixture(d)
    X = d["X_seeded"].copy()
    X[3] = np.nan
    with pytest.raises(TDGLError, match="non-finite"):
        tb.trapezoidal(X, dev.params, dev.idx, tb.FieldSchedule(dev.applied_field, dev.params, dev.idx, 1.0),
                       0.0, 1.0, 0.1, progress=False)


def test_generic_callable_contract(tb):
    # the reference's own solver tests use plain Python callables
    b = np.array([1.0, 2.0], dtype=np.complex128)
    x = tb.tgcr_matrix_free_trap(lambda v: v, np.zeros(2, dtype=np.complex128), b, dt=0.0, tol=1e-8)
    np.testing.assert_allclose(x, b, atol=1e-5)
    x0 = np.array([1.0, 2.0], dtype=np.complex128)
    xs, ok, it = tb.newton_gcr_trap(lambda v: np.zeros_like(v), x0, x0.copy(), dt=1.0, tol_f=1e-6, tol_dx=1e-6)
    assert ok
    np.testing.assert_allclose(xs, x0, atol=1e-4)


@pytest.mark.parametrize("periodic", [(False, False, False), (True, False, True)])
def test_fused_arnoldi_across_tiles(tb, periodic):
    """The fused Arnoldi kernel (analytic products, GMRES) on a grid of several
    x/y tiles and single-plane z-chunks, with a hole: its trajectory agrees
    with the finite-difference graph path and the persistent GCR stepper at
    the Newton tolerance level."""
    px, py, pz = periodic
    p = tb.SimulationParameters(Nx=70, Ny=20, Nz=12, hx=0.5, hy=0.5, hz=0.5, kappa=2.0,
                                periodic_x=px, periodic_y=py, periodic_z=pz)
    dev = tb.Device(p, applied_field=tb.AppliedField(Bz=0.4, By=0.1, t_on_fraction=1.0))
    dev.add_hole([(10.0, 3.0), (14.0, 3.0), (14.0, 6.0), (10.0, 6.0)], z_range=(2, 7))
    x0 = dev.initial_state()
    rng = np.random.default_rng(5)
    n = x0.psi.shape[0]
    x0.psi += 0.05 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    kw = dict(t_start=0.0, t_stop=0.3, dt=0.1, method="trapezoidal", x0=x0, progress=False, log_metadata=False,
              newton_tol_f=1e-8, newton_tol_dx=1e-3, tol_gcr=1e-6, precision="fp64")
    fused = tb.solve(dev, jvp="analytic", krylov="gmres", **kw)
    fd = tb.solve(dev, jvp="fd", krylov="gmres", **kw)
    gcr = tb.solve(dev, jvp="analytic", krylov="gcr", **kw)
    assert np.array_equal(fused.times, fd.times)
    assert np.max(np.abs(fused.states - fd.states)) < 1e-7
    assert np.max(np.abs(fused.states - gcr.states)) < 1e-7
    mixed = tb.solve(dev, **{**kw, "precision": "mixed"})
    p64 = np.abs(fused.psi(-1)) ** 2
    assert np.linalg.norm(np.abs(mixed.psi(-1)) ** 2 - p64) / np.linalg.norm(p64) < 1e-6


@pytest.mark.parametrize("kappa", [3.0, 4.0])
def test_mixed_precision_stiff_kappa(tb, kappa):
    """Large kappa^2 dt / h^2 (a stiff phi block, long Krylov solves): the
    FP32 Arnoldi basis stays in range and the mixed stepper tracks FP64."""
    p = tb.SimulationParameters(Nx=20, Ny=12, Nz=4, hx=0.5, hy=0.5, hz=0.5, kappa=kappa)
    dev = tb.Device(p, applied_field=tb.AppliedField(Bz=0.6, t_on_fraction=1.0))
    dev.add_hole([(3.0, 2.0), (5.0, 2.0), (5.0, 4.0), (3.0, 4.0)])
    x0 = dev.initial_state()
    rng = np.random.default_rng(7)
    n = x0.psi.shape[0]
    x0.psi += 0.01 * (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * dev.material.interior_sc_mask
    kw = dict(t_start=0.0, t_stop=0.5, dt=0.1, method="trapezoidal", x0=x0, progress=False, log_metadata=False,
              newton_tol_f=1e-8, newton_tol_dx=1e-3, tol_gcr=1e-6)
    ref = tb.solve(dev, precision="fp64", **kw)
    mix = tb.solve(dev, precision="mixed", **kw)
    assert np.array_equal(ref.times, mix.times)
    p_ref = np.abs(ref.psi(-1)) ** 2
    p_mix = np.abs(mix.psi(-1)) ** 2
    assert np.linalg.norm(p_mix - p_ref) / np.linalg.norm(p_ref) < 1e-6


def _oracle_run(dev, x0, fld, t_stop, **kw):
    from oracle import tdgl_oracle as orc
    g = orc.make_grid(dev.params, dev.idx, dev.material)
    return orc.trapezoidal(x0, g, fld, 0.0, t_stop, 0.1, **kw)


@pytest.mark.parametrize("mode", ["ramp", "field_func"])
def test_field_schedules_match_oracle(tb, mode):
    """A ramped field (evaluated on the device each step) and a Python
    field_func (evaluated on the host each step) against the oracle."""
    from oracle import tdgl_oracle as orc
    p = tb.SimulationParameters(Nx=10, Ny=8, Nz=4, hx=0.5, hy=0.5, hz=0.5, kappa=2.0)
    t_stop = 0.6
    if mode == "ramp":
        af = tb.AppliedField(Bx=0.1, By=0.05, Bz=0.6, t_on_fraction=0.9, ramp=True, ramp_fraction=0.5)
        fld = orc.field_schedule(Bx=0.1, By=0.05, Bz=0.6, t_on_fraction=0.9, ramp=True, ramp_fraction=0.5,
                                 t_stop=t_stop)
    else:
        def ff(t, ts):
            return 0.05 * t, 0.0, 0.4 + 0.3 * np.sin(3.0 * t / ts)
        af = tb.AppliedField(field_func=ff)
        fld = lambda t: ff(t, t_stop)  # noqa: E731
    dev = tb.Device(p, applied_field=af)
    dev.add_hole([(1.5, 1.0), (3.0, 1.0), (3.0, 2.5), (1.5, 2.5)])
    x0 = dev.initial_state()
    rng = np.random.default_rng(11)
    n = x0.psi.shape[0]
    x0.psi += 0.02 * (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * dev.material.interior_sc_mask
    kw = dict(newton_tol_f=1e-8, newton_tol_dx=1e-3, tol_gcr=1e-6)
    sol = tb.solve(dev, t_start=0.0, t_stop=t_stop, dt=0.1, method="trapezoidal", x0=x0.data, progress=False,
                   log_metadata=False, **kw)
    times, hist = _oracle_run(dev, x0.data, fld, t_stop, **kw)
    assert np.allclose(sol.times, times, rtol=0, atol=1e-14)
    assert np.max(np.abs(sol.states - hist)) < 1e-7
