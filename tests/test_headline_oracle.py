"""Parity at the benchmarked size against the oracle.

The workload is the one ``bench.py`` times: a 128x128x32-cell film with the
centred 32x32-node hole through all planes (499,999 interior nodes,
1,999,996 state entries), kappa 2, Bz 0.5, seeded psi0 noise.  Small-grid
goldens cannot show the tile seams of the 127-node rows or the hole at this
size; these tests compare the CUDA path with the oracle on the same seeded
state:

* FP64 RHS (with the applied-field face offsets) against ``oracle.eval_f``
  (src/tdgl3d/physics/rhs.py:147-239): 1e-12 relative (summation order only).
* One trapezoidal step with the field on (t = 0.1 -> 0.2; the schedule is 0 at
  t = 0, src/tdgl3d/physics/applied_field.py:42-56) against
  ``oracle.trapezoidal(max_steps=1)`` (src/tdgl3d/solvers/integrators.py:150-197):
  the FP64 finite-difference stepper with the reference's GCR and with GMRES,
  and the mixed-precision stepper (FP32 Krylov vectors, analytic products,
  polynomial preconditioner).  Each Newton solve stops at ||g||_inf <= 1e-8, so
  every stepper lands within ~1e-8 of the exact step: 1e-7 absolute on the
  state, and the north star's 1e-6 relative L2 bound on |psi|^2.

The oracle's step takes about 40 s of one host core; it is computed once.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

T0, DT = 0.1, 0.1


@pytest.fixture(scope="module")
def headline():
    import bench
    from oracle import tdgl_oracle as orc
    assert torch.cuda.is_available()
    dev, x0 = bench.build_device()
    w = bench.WORKLOAD
    og = orc.make_grid(dev.params, dev.idx, dev.material)
    fld = orc.field_schedule(Bz=w["Bz"], t_on_fraction=1.0, t_stop=w["t_stop"])
    kw = dict(newton_tol_f=w["tol_f"], newton_tol_dx=w["tol_dx"], tol_gcr=w["tol_gcr"], eps_mf=w["eps_mf"])
    times, hist = orc.trapezoidal(x0, og, fld, T0, w["t_stop"], DT, max_steps=1, **kw)
    assert abs(times[-1] - (T0 + DT)) < 1e-12
    return dict(dev=dev, x0=x0, w=w, og=og, kw=kw, x1=hist[:, -1], B=fld(T0))


def _psi2_rel(x, ref, n):
    a, b = np.abs(x[:n]) ** 2, np.abs(ref[:n]) ** 2
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_eval_f_at_headline_size(headline):
    from nanowire_tdgl_b200.engine import grid_for
    from oracle import tdgl_oracle as orc
    h = headline
    dev = h["dev"]
    g = grid_for(dev.params, dev.idx, dev.material)
    rng = np.random.default_rng(11)
    n = dev.params.n_interior
    X = h["x0"].copy()
    # links away from zero, so that every Peierls factor and supercurrent term is exercised
    X[n:] = 0.3 * rng.standard_normal(X.size - n) + 0j
    for B in [(0.0, 0.0, h["w"]["Bz"]), (0.2, -0.3, 0.5)]:
        F = g.eval_f_ref(X, B).cpu().numpy()
        want = orc.eval_f(X, h["og"], *B)
        rel = np.max(np.abs(F - want)) / np.max(np.abs(want))
        assert rel < 1e-12, f"B={B}: relative max error {rel:.3e}"


@pytest.mark.parametrize("precision,krylov", [("fp64", "gcr"), ("fp64", "gmres"), ("mixed", "gmres")])
def test_one_step_at_headline_size(headline, precision, krylov):
    import nanowire_tdgl_b200 as tb
    h = headline
    dev, w = h["dev"], h["w"]
    p = dev.params
    sched = tb.FieldSchedule(dev.applied_field, p, dev.idx, w["t_stop"])
    jvp = "fd" if precision == "fp64" else "analytic"
    times, hist = tb.trapezoidal(h["x0"], p, dev.idx, sched, T0, T0 + DT, DT, material=dev.material,
                                 progress=False, precision=precision, jvp=jvp, krylov=krylov, **h["kw"])
    assert len(times) == 2 and abs(times[-1] - (T0 + DT)) < 1e-12
    x1 = hist[:, -1]
    err = float(np.max(np.abs(x1 - h["x1"])))
    rel = _psi2_rel(x1, h["x1"], p.n_interior)
    assert err < 1e-7, f"{precision}/{krylov}: max |x - oracle| = {err:.3e}"
    assert rel < 1e-6, f"{precision}/{krylov}: |psi|^2 relative L2 = {rel:.3e}"


def test_eval_f_at_trilayer_size():
    """The 256x256x64 S/I/S trilayer with its 64x64 hole (4,096,575 interior
    nodes; the large configuration of the bench's forms): FP64 RHS against
    the oracle at 1e-12 relative, with links away from zero."""
    import bench
    from nanowire_tdgl_b200.engine import grid_for
    from oracle import tdgl_oracle as orc
    dev, x0 = bench.trilayer_device()
    og = orc.make_grid(dev.params, dev.idx, dev.material)
    g = grid_for(dev.params, dev.idx, dev.material)
    n = dev.params.n_interior
    X = x0.copy()
    X[n:] = 0.3 * np.random.default_rng(13).standard_normal(X.size - n) + 0j
    B = (0.0, 0.0, bench.TRI["Bz"])
    F = g.eval_f_ref(X, B).cpu().numpy()
    want = orc.eval_f(X, og, *B)
    rel = np.max(np.abs(F - want)) / np.max(np.abs(want))
    assert rel < 1e-12, f"relative max error {rel:.3e}"
