"""Batched form against the reference: the reference's golden trapezoidal
trajectories (``trap_*`` fixtures, made by tdgl3d's own ``trapezoidal``)
stepped together as one batch, each instance checked against the states the
reference saved.

The batch follows each device's ``AppliedField`` schedule
(``field_schedule=True``; zero field at t = 0 like the reference's first
step).  Every fixture uses dt 0.1 and the Newton/Krylov tolerances the batch
is given; the states after steps 2 and 5 are compared wherever the fixture
saved them.  Tolerance: 1e-6 absolute on the state and 1e-6 relative L2 on
|psi|^2.  Each step's Newton iterate is within its ||g||_inf <= 1e-8 test of
the reference's (src/tdgl3d/solvers/newton.py:76-120), so five steps stay
near 1e-7 whatever the Krylov form; an instance stepped with another's field,
state or clock is off by far more.
"""

import numpy as np
import pytest

from conftest import device_from_fixture, golden, golden_names

TRAPS = golden_names("trap_")
DT = 0.1
TOL = dict(newton_tol_f=1e-8, newton_tol_dx=1e-3, tol_gcr=1e-6, eps_mf=1e-4)


def _batch_inputs():
    devs, xs, refs = [], [], []
    for name in TRAPS:
        d = golden(name)
        assert float(d["dt"]) == DT
        assert (float(d["kw_newton_tol_f"]), float(d["kw_newton_tol_dx"]), float(d["kw_tol_gcr"]),
                float(d["kw_eps_mf"])) == tuple(TOL.values()), name
        devs.append(device_from_fixture(golden("case_" + name[len("trap_"):])))
        xs.append(d["x0"])
        refs.append(d)
    return devs, xs, refs


def _saved(d, step):
    j = np.nonzero(d["saved_steps"] == step)[0]
    return d["states"][:, j[0]] if j.size else None


def test_fixtures_cover_both_checkpoints():
    """Every trajectory saved step 2, all but the 101-step one step 5."""
    refs = [golden(n) for n in TRAPS]
    assert len(refs) >= 5
    assert all(_saved(d, 2) is not None for d in refs)
    assert sum(_saved(d, 5) is not None for d in refs) >= len(refs) - 1


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_reference_trajectories(precision):
    import nanowire_tdgl_b200 as tb
    devs, xs, refs = _batch_inputs()
    b = tb.BatchedTrapezoidal(devs, xs, DT, t_stop=1.0, precision=precision, kmax=96, n_streams=4,
                              field_schedule=True, **TOL)
    b.set_shape(2, 1)
    done = 0
    for step in (2, 5):
        b.step(step - done)
        done = step
        assert all(abs(t - DT * step) < 1e-12 for t in b.t)
        checked = 0
        for name, dev, d, x in zip(TRAPS, devs, refs, b.states()):
            ref = _saved(d, step)
            if ref is None:
                continue
            err = np.max(np.abs(x - ref))
            assert err < 1e-6, (name, step, err)
            n = ref.size // (4 if dev.params.is_3d else 3)
            p, q = np.abs(x[:n]) ** 2, np.abs(ref[:n]) ** 2
            assert np.linalg.norm(p - q) / np.linalg.norm(q) < 1e-6, (name, step)
            checked += 1
        assert checked >= len(TRAPS) - (step == 5)
