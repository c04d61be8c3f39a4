"""Pin the CPU oracle (oracle/tdgl_oracle.py) to the reference's own outputs.

The oracle is test infrastructure: it is the checker for the CUDA path, so
before trusting it, it must reproduce every golden vector recorded from the
reference (tests/golden/make_golden.py)."""

import numpy as np
import pytest

from conftest import device_from_fixture, golden, golden_names

from oracle import tdgl_oracle as orc

CASES = golden_names("case_")
RTOL_RHS = 1e-12   # FP64 RHS, different summation order from the CSR matvec


def _grid(d):
    dev = device_from_fixture(d)
    return dev, orc.make_grid(dev.params, dev.idx, dev.material)


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("name", CASES)
def test_oracle_eval_f(name):
    d = golden(name)
    dev, g = _grid(d)
    bx, by, bz = d["B"]
    F = orc.eval_f(d["X_seeded"], g, bx, by, bz)
    assert _rel(F, d["F_seeded"]) < RTOL_RHS
    if "X_random" in d:
        F = orc.eval_f(d["X_random"], g, bx, by, bz)
        assert _rel(F, d["F_random"]) < RTOL_RHS
        F0 = orc.eval_f(d["X_random"], g, 0.0, 0.0, 0.0)
        assert _rel(F0, d["F_random_b0"]) < RTOL_RHS


@pytest.mark.parametrize("name", ["solver_3d_basic", "solver_3d_hole", "solver_2d_basic"])
def test_oracle_solvers(name):
    d = golden(name)
    case = golden("case_" + name[len("solver_"):])
    dev, g = _grid(case)
    f = orc.make_rhs(g, *case["B"])
    dt = float(d["dt"])
    x = orc.tgcr_trap(f, d["x_lin"], d["b"], dt, tol=float(d["tgcr_tol"]))
    assert _rel(x, d["tgcr_x"]) < 1e-6
    xn, ok, it = orc.newton_trap(f, d["x_pred"], d["gamma"], dt, tol_f=1e-8, tol_dx=1e-3,
                                 max_iter=20, tol_gcr=1e-6)
    assert ok == bool(d["newton_converged"]) and it == int(d["newton_iters"])
    assert np.max(np.abs(xn - d["newton_x"])) < 1e-8


@pytest.mark.parametrize("name", [n for n in golden_names("trap_") if n != "trap_config1"])
def test_oracle_trapezoidal_short(name):
    d = golden(name)
    case = golden("case_" + name[len("trap_"):])
    dev, g = _grid(case)
    bx, by, bz = case["B"]
    fld = orc.field_schedule(bx, by, bz, t_on_fraction=1.0, t_stop=float(d["t_stop"]))
    times, hist = orc.trapezoidal(d["x0"], g, fld, 0.0, float(d["t_stop"]), float(d["dt"]),
                                  newton_tol_f=1e-8, newton_tol_dx=1e-3, tol_gcr=1e-6)
    assert np.array_equal(times, d["times"])
    err = np.max(np.abs(hist[:, d["saved_steps"]] - d["states"]))
    assert err < 1e-7, err


def test_oracle_euler():
    d = golden("euler_3d_hole")
    case = golden("case_3d_hole")
    dev, g = _grid(case)
    fld = orc.field_schedule(*case["B"], t_on_fraction=1.0, t_stop=float(d["t_stop"]))
    times, hist = orc.forward_euler(d["x0"], g, fld, 0.0, float(d["t_stop"]), float(d["dt"]))
    assert np.allclose(times, d["times"], rtol=0, atol=1e-15)
    assert _rel(hist[:, d["saved_steps"]], d["states"]) < 1e-11


@pytest.mark.parametrize("name", [n for n in golden_names("trap_") if n != "trap_config1"])
def test_oracle_observables(name):
    d = golden(name)
    case = golden("case_" + name[len("trap_"):])
    dev, g = _grid(case)
    X = d["states"][:, -1]
    assert np.allclose(orc.psi_squared(X, g), d["psi2"], rtol=0, atol=1e-14)
    bx, by, bz = case["B"]   # t_on_fraction = 1: the field is on at t_stop
    B = orc.bfield(X, g, bx, by, bz)
    for mine, ref in zip(B, (d["Bx"], d["By"], d["Bz"])):
        assert np.allclose(mine, ref, rtol=0, atol=1e-12)
    J = orc.supercurrent_density(X, g)
    for mine, ref in zip(J, (d["Jx"], d["Jy"], d["Jz"])):
        assert np.allclose(mine, ref, rtol=0, atol=1e-13)
