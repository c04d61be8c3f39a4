"""Queued step-graph launches: tdgl_trap_launch followed by
tdgl_trap_launch_next continuations equal one blocking tdgl_trap_run over the
same steps, bit for bit (the same graph and reductions; the continuation
takes the clock the previous launch left on the device), and misuse is
refused on the host.  trapezoidal() queues its launches this way; its
trajectories are checked against the reference in test_gpu_parity.py."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup(precision):
    import nanowire_tdgl_b200 as tb
    from nanowire_tdgl_b200 import _lib as L
    from nanowire_tdgl_b200.engine import DeviceGrid
    p = tb.SimulationParameters(Nx=30, Ny=16, Nz=8, hx=0.5, hy=0.5, hz=0.5, kappa=2.0)
    dev = tb.Device(p, applied_field=tb.AppliedField(Bz=0.5, t_on_fraction=1.0))
    dev.add_hole([(6.0, 3.0), (9.0, 3.0), (9.0, 5.0), (6.0, 5.0)])
    x0 = dev.initial_state()
    rng = np.random.default_rng(12)
    n = p.n_interior
    x0.psi[:] += 0.01 * (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * dev.material.interior_sc_mask
    opts = L.TrapOpts(0.75, 0.1, 1e-8, 1e-8, 1e-3, 1e-6, 1e-4, 20, 0, 1, L.TDGL_JVP_ANALYTIC)
    fld = L.Field(0.0, 0.0, 0.5, 1.0, 0.5, 0.75, 0, 0)
    mk = lambda: DeviceGrid(p, dev.idx, dev.material, precision, 32)  # noqa: E731
    return mk, x0.data, opts, fld


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_continuations_equal_one_run(precision):
    from nanowire_tdgl_b200 import _lib as L
    mk, x0, opts, fld = _setup(precision)
    ref = mk()
    xr = ref.pack(x0)
    rc, t_ref, cur_ref, st_ref = ref.trap_run(xr, 0.0, 0.1, 10, opts, fld)
    assert rc == L.TDGL_OK and st_ref["steps"] == 8      # t_stop 0.75: seven full steps and a 0.05 step
    g = mk()
    x = g.pack(x0)
    s = torch.cuda.current_stream()
    g.trap_launch(x, 0.0, 0.1, 3, opts, fld, s)
    g.trap_launch_next(x, 3, opts, fld, s)
    clocks, steps = [], 0
    rc, t, cur, st = g.trap_collect()
    assert rc == L.TDGL_OK and st["steps"] == 3
    clocks.append(t)
    g.trap_launch_next(x, 3, opts, fld, s)
    for _ in range(2):
        rc, t, cur, st = g.trap_collect()
        assert rc == L.TDGL_OK
        steps += st["steps"]
        clocks.append(t)
    assert steps == 5                                     # three more, then the last two up to t_stop
    assert abs(clocks[0] - 0.3) < 1e-12 and t == t_ref and cur == cur_ref
    assert torch.equal(x, xr)
    # a further continuation at t_stop runs no step
    g.trap_launch_next(x, 3, opts, fld, s)
    rc, t2, _, st = g.trap_collect()
    assert rc == L.TDGL_OK and st["steps"] == 0 and t2 == t
    assert torch.equal(x, xr)


def test_queue_misuse_is_refused():
    from nanowire_tdgl_b200 import _lib as L
    mk, x0, opts, fld = _setup("mixed")
    g = mk()
    x = g.pack(x0)
    s = torch.cuda.current_stream()
    with pytest.raises(L.TDGLError):                      # nothing to continue yet
        g.trap_launch_next(x, 1, opts, fld, s)
    rc, _, _, _ = g.trap_collect()                        # nothing to collect
    assert rc == L.TDGL_EINVAL
    g.trap_launch(x, 0.0, 0.1, 1, opts, fld, s)
    g.trap_launch_next(x, 1, opts, fld, s)
    with pytest.raises(L.TDGLError):                      # two already queued
        g.trap_launch_next(x, 1, opts, fld, s)
    with pytest.raises(L.TDGLError):                      # settings wait for the queue
        g.set_poly(3)
    for _ in range(2):
        rc, _, _, _ = g.trap_collect()
        assert rc == L.TDGL_OK
