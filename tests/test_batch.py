"""Batched form: instances stepped concurrently give exactly the states of
stepping them one after another with the same launch shapes; stream
assignment and block-count rules checked on the host."""

import numpy as np
import pytest


def _instances(n=5, seed=0, variety=False):
    """Seeded instances of uneven size, kappa, field and holes; with variety,
    the first two are a trilayer and a periodic film."""
    import nanowire_tdgl_b200 as tb
    rng = np.random.default_rng(seed)
    devs, xs = [], []
    for q in range(n):
        Nx, Ny = (int(v) for v in rng.choice([12, 16, 20, 24], 2))
        Nz = int(rng.choice([1, 4, 6]))
        kappa = float(rng.uniform(1.5, 4))
        field = tb.AppliedField(Bz=float(rng.uniform(0.1, 1.0)), t_on_fraction=1.0)
        if variety and q == 0:
            p = tb.SimulationParameters(Nx=Nx, Ny=Ny, Nz=7, hx=0.5, hy=0.5, hz=0.5, kappa=kappa)
            tri = tb.Trilayer(tb.Layer(3, kappa), tb.Layer(2, kappa, is_superconductor=False), tb.Layer(2, kappa))
            d = tb.Device(p, applied_field=field, trilayer=tri)
        elif variety and q == 1:
            p = tb.SimulationParameters(Nx=Nx, Ny=Ny, Nz=Nz, hx=0.5, hy=0.5, hz=0.5, kappa=kappa, periodic_x=True)
            d = tb.Device(p, applied_field=field)
        else:
            p = tb.SimulationParameters(Nx=Nx, Ny=Ny, Nz=Nz, hx=0.5, hy=0.5, hz=0.5, kappa=kappa)
            d = tb.Device(p, applied_field=field)
        if q % 2:
            i0, j0 = int(rng.integers(3, Nx - 8)), int(rng.integers(3, Ny - 8))
            s = int(rng.integers(3, 6))
            d.add_hole([(0.5 * i0, 0.5 * j0), (0.5 * (i0 + s), 0.5 * j0), (0.5 * (i0 + s), 0.5 * (j0 + s)),
                        (0.5 * i0, 0.5 * (j0 + s))])
        x = d.initial_state()
        m = x.psi.shape[0]
        x.psi[:] += 0.02 * (rng.standard_normal(m) + 1j * rng.standard_normal(m))
        devs.append(d)
        xs.append(x.data.copy())
    return devs, xs


def test_stream_assignment_balances_work():
    from nanowire_tdgl_b200.batch import assign_streams
    sizes = [135375, 2883, 50000, 50000, 9000, 120000, 4000, 60000]
    queues, order = assign_streams(sizes, 3)
    assert sorted(i for q in queues for i in q) == list(range(len(sizes)))
    assert sorted(i for _, i in order) == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in q) for q in queues]
    assert max(loads) <= sum(sizes) / 3 + max(sizes)
    assert queues[0][0] == 0                        # largest first
    assert [i for _, i in order[:3]] == [q[0] for q in queues]   # first of every stream first
    assert all(order.index((s, q[r])) < order.index((s, q[r + 1])) for s, q in enumerate(queues)
               for r in range(len(q) - 1))
    assert len(assign_streams(sizes, 100)[0]) == len(sizes)


def test_block_rule():
    from nanowire_tdgl_b200.batch import launch_blocks
    assert launch_blocks(10_000, None, 148) == (8 * 148, 5 * 148)
    assert launch_blocks(2883, 1, 148) == (12, 8)
    assert launch_blocks(2883, 16, 148) == (1, 1)
    assert launch_blocks(10 ** 8, 1, 148) == (8 * 148, 5 * 148)


def test_instance_field_constant_and_schedule():
    """Constant field by default; with field_schedule the AppliedField's
    schedule against t_stop, as the device evaluates it for ``solve``."""
    import nanowire_tdgl_b200 as tb
    from nanowire_tdgl_b200.batch import instance_field
    af = tb.AppliedField(Bx=0.1, By=-0.2, Bz=0.5, t_on_fraction=0.8, ramp=True, ramp_fraction=0.25)
    c = instance_field(af, 1e30, False)
    assert (c.Bx, c.By, c.Bz, c.constant) == (0.1, -0.2, 0.5, 1)
    s = instance_field(af, 2.0, True)
    assert (s.Bx, s.By, s.Bz) == (0.1, -0.2, 0.5)
    assert (s.constant, s.t_field_stop, s.t_on_fraction, s.ramp_fraction, s.ramp) == (0, 2.0, 0.8, 0.25, 1)
    with pytest.raises(ValueError):
        instance_field(af, float("inf"), True)
    with pytest.raises(ValueError):
        instance_field(tb.AppliedField(field_func=lambda t, ts: (0.0, 0.0, t)), 1.0, True)
    assert instance_field(tb.AppliedField(field_func=lambda t, ts: (0.0, 0.0, t)), 1.0, False).constant == 1


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("shape", [(None, -1), (2, 0), (2, 1)])
def test_batched_equals_sequential(precision, shape):
    import nanowire_tdgl_b200 as tb
    devs, xs = _instances()
    a = tb.BatchedTrapezoidal(devs, xs, 0.1, precision=precision, kmax=96, n_streams=3)
    a.set_shape(*shape)
    a.step(3)
    sa = a.states()
    ta, tot_a = list(a.t), dict(a.totals)
    b = tb.BatchedTrapezoidal(devs, xs, 0.1, precision=precision, kmax=96)
    b.set_shape(*shape)
    b.step_sequential(3)
    for u, v in zip(sa, b.states()):
        assert np.array_equal(u, v)
    assert ta == b.t and tot_a == b.totals
    assert all(abs(t - 0.3) < 1e-12 for t in ta)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batched_trilayer_and_periodic_instances(precision):
    """A trilayer (psi relaxed in the insulator) and a periodic film in the
    batch: concurrent steps equal the one-by-one steps bit for bit."""
    import nanowire_tdgl_b200 as tb
    devs, xs = _instances(4, seed=3, variety=True)
    a = tb.BatchedTrapezoidal(devs, xs, 0.1, precision=precision, kmax=96, n_streams=4)
    a.set_shape(2, 1)
    a.step(2)
    b = tb.BatchedTrapezoidal(devs, xs, 0.1, precision=precision, kmax=96)
    b.set_shape(2, 1)
    b.step_sequential(2)
    for u, v in zip(a.states(), b.states()):
        assert np.array_equal(u, v)
    assert a.totals == b.totals


@pytest.mark.gpu
def test_small_launch_shape_matches_default_within_tolerance():
    """Other block counts change only the reduction partition: tightly
    converged states agree with the default shape's to rounding."""
    import nanowire_tdgl_b200 as tb
    devs, xs = _instances(3, seed=2)
    kw = dict(precision="fp64", kmax=96, newton_tol_f=1e-12, newton_tol_dx=1e-10, tol_gcr=1e-11)
    a = tb.BatchedTrapezoidal(devs, xs, 0.1, **kw)
    a.set_shape(None)
    a.step(2)
    sa = a.states()
    a2 = tb.BatchedTrapezoidal(devs, xs, 0.1, **kw)
    a2.set_shape(16, 1)
    a2.step(2)
    for u, v in zip(sa, a2.states()):
        assert np.max(np.abs(u - v)) < 1e-9


@pytest.mark.gpu
def test_default_shape_after_fused_shape_is_the_default():
    """Setting the default form (fused -1) after a fused shape restores the
    default, so a context that went through the autotuner steps like a fresh
    one with the same shape."""
    import nanowire_tdgl_b200 as tb
    devs, xs = _instances(3, seed=4)
    a = tb.BatchedTrapezoidal(devs, xs, 0.1, kmax=96)
    snap = a.snapshot()
    a.set_shape(4, 1)
    a.step(1)
    a.set_shape(None, -1)
    a.restore(snap)
    a.step(2)
    b = tb.BatchedTrapezoidal(devs, xs, 0.1, kmax=96)
    b.set_shape(None, -1)
    b.step_sequential(2)
    for u, v in zip(a.states(), b.states()):
        assert np.array_equal(u, v)


@pytest.mark.gpu
def test_autotune_keeps_a_candidate_and_restores_states():
    import nanowire_tdgl_b200 as tb
    devs, xs = _instances(4, seed=1)
    a = tb.BatchedTrapezoidal(devs, xs, 0.1, kmax=96)
    x_before = [x.clone() for x in a.x]
    times = a.autotune(((None, -1), (4, 1)), steps=1)
    assert a.best in times and a.shape == a.best
    assert all(np.array_equal(u.cpu().numpy(), v.cpu().numpy()) for u, v in zip(x_before, a.x))
    assert a.t == [0.0] * 4 and a.totals["steps"] == 0
    a.step(2)
    b = tb.BatchedTrapezoidal(devs, xs, 0.1, kmax=96)
    b.set_shape(*a.best)
    b.step_sequential(2)
    for u, v in zip(a.states(), b.states()):
        assert np.array_equal(u, v)


@pytest.mark.gpu
def test_async_entry_points_reject_misuse():
    """tdgl_trap_collect with nothing launched, a second launch before the
    collect, and block counts outside [1, 8 x SMs] are refused with
    TDGL_EINVAL; the context stays usable."""
    import ctypes as C
    import torch
    import nanowire_tdgl_b200 as tb
    from nanowire_tdgl_b200 import _lib as L
    devs, xs = _instances(1, seed=5)
    a = tb.BatchedTrapezoidal(devs, xs, 0.1, kmax=96)
    g = a.grids[0]
    tt, dd, st = C.c_double(0.0), C.c_double(0.0), L.Stats()
    assert g.lib.tdgl_trap_collect(g.handle, C.byref(tt), C.byref(dd), C.byref(st)) == L.TDGL_EINVAL
    assert g.lib.tdgl_ctx_set_blocks(g.handle, 0, 10, -1) == L.TDGL_EINVAL
    assert g.lib.tdgl_ctx_set_blocks(g.handle, 10, 8 * a.sms + 1, -1) == L.TDGL_EINVAL
    s = a.streams[0]
    g.trap_launch(a.x[0], 0.0, 0.1, 1, a.opts, a.fields[0], s)
    rc = g.lib.tdgl_trap_launch(g.handle, C.c_void_p(a.x[0].data_ptr()), 0.0, 0.1, 1, C.byref(a.opts),
                                C.byref(a.fields[0]), C.c_void_p(s.cuda_stream))
    assert rc == L.TDGL_EINVAL
    assert g.lib.tdgl_ctx_set_blocks(g.handle, 10, 10, -1) == L.TDGL_EINVAL     # a launch is pending
    rc = g.lib.tdgl_trap_run(g.handle, C.c_void_p(a.x[0].data_ptr()), C.byref(C.c_double(0.0)),
                             C.byref(C.c_double(0.1)), 1, C.byref(a.opts), C.byref(a.fields[0]), C.byref(L.Stats()),
                             C.c_void_p(s.cuda_stream))
    assert rc == L.TDGL_EINVAL                                                    # shares the workspace
    s.synchronize()
    rc, t, cur, stats = g.trap_collect()
    assert rc == L.TDGL_OK and abs(t - 0.1) < 1e-12 and stats["steps"] == 1
    a.t[0], a.cur[0] = t, cur
    a.step(1)
    assert abs(a.t[0] - 0.2) < 1e-12


@pytest.mark.gpu
def test_single_instance_and_more_streams_than_instances():
    import nanowire_tdgl_b200 as tb
    devs, xs = _instances(1, seed=6)
    a = tb.BatchedTrapezoidal(devs, xs, 0.1, kmax=96, n_streams=8)
    assert len(a.streams) == 1
    a.step(2)
    b = tb.BatchedTrapezoidal(devs, xs, 0.1, kmax=96)
    b.step_sequential(2)
    assert np.array_equal(a.states()[0], b.states()[0])
