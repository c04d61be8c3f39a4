"""The device's bounded waits and loop caps run out, report their status, and
leave the context usable.

Every wait inside a kernel is bounded by the context's wait limit
(``tdgl_ctx_set_limits``): the persistent GCR kernel's grid barrier and the
staged-copy waits of the TMA-staged stencil.  A limit of 1 ns makes the first
wait that is not already complete give up; the kernel stops (the stencil
first waits, with its own bound, for the copies it has in flight), the call
returns TDGL_ETIMEOUT and later kernels of the launch return at once.  The
loop cap bounds the conditional-loop iterations of one step-graph launch.
Restoring the defaults, the same context then steps exactly as a fresh one.
Kernels launched outside the graph (the Arnoldi-step probe) record a
failure's status without touching the graph's conditional nodes.
The reference has no device waits; its failure conventions (a failed solve
is an exception, src/tdgl3d/solvers/integrators.py:186-197) are kept by the
Python layer for the codes it maps.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup(precision, krylov="gmres"):
    import nanowire_tdgl_b200 as tb
    from nanowire_tdgl_b200 import _lib as L
    from nanowire_tdgl_b200.engine import DeviceGrid
    p = tb.SimulationParameters(Nx=40, Ny=18, Nz=10, hx=0.5, hy=0.5, hz=0.5, kappa=2.0)
    dev = tb.Device(p, applied_field=tb.AppliedField(Bz=0.5, t_on_fraction=1.0))
    dev.add_hole([(8.0, 3.0), (11.0, 3.0), (11.0, 6.0), (8.0, 6.0)])
    x0 = dev.initial_state()
    rng = np.random.default_rng(2)
    n = p.n_interior
    x0.psi[:] += 0.01 * (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * dev.material.interior_sc_mask
    jvp = L.TDGL_JVP_FD if precision == "fp64" and krylov == "gcr" else L.TDGL_JVP_ANALYTIC
    opts = L.TrapOpts(5.0, 0.1, 1e-8, 1e-8, 1e-3, 1e-6, 1e-4, 20, 0, 1, jvp)
    fld = L.Field(0.0, 0.0, 0.5, 1.0, 0.5, 5.0, 0, 0)
    mk = lambda: DeviceGrid(p, dev.idx, dev.material, precision, 32, krylov)  # noqa: E731
    return mk, x0.data, opts, fld


def _run(g, x0, opts, fld, steps=2):
    x = g.pack(x0)
    rc, t, cur, st = g.trap_run(x, 0.1, 0.1, steps, opts, fld)
    torch.cuda.synchronize()
    return rc, x


@pytest.mark.parametrize("precision,krylov", [("mixed", "gmres"), ("fp64", "gcr")])
def test_wait_limit_runs_out_and_context_recovers(precision, krylov):
    from nanowire_tdgl_b200 import _lib as L
    mk, x0, opts, fld = _setup(precision, krylov)
    ref = mk()
    rc, want = _run(ref, x0, opts, fld)
    assert rc == L.TDGL_OK
    g = mk()
    g.set_limits(wait_ns=1)
    rc, _ = _run(g, x0, opts, fld)
    assert rc == L.TDGL_ETIMEOUT
    g.set_limits()
    rc, got = _run(g, x0, opts, fld)
    assert rc == L.TDGL_OK
    assert torch.equal(got, want)


def test_loop_cap_runs_out_and_context_recovers():
    from nanowire_tdgl_b200 import _lib as L
    mk, x0, opts, fld = _setup("mixed")
    ref = mk()
    rc, want = _run(ref, x0, opts, fld)
    assert rc == L.TDGL_OK
    g = mk()
    g.set_limits(loop_cap=1)
    rc, _ = _run(g, x0, opts, fld)
    assert rc == L.TDGL_ETIMEOUT
    g.set_limits()
    rc, got = _run(g, x0, opts, fld)
    assert rc == L.TDGL_OK
    assert torch.equal(got, want)


def test_staged_stencil_wait_limit():
    """The TMA-staged product alone on the 128x128x32 bench device (384
    blocks issuing their first copies together): a 1 ns wait limit gives
    TDGL_ETIMEOUT, the default limit the exact product again."""
    import bench
    from nanowire_tdgl_b200 import _lib as L
    from nanowire_tdgl_b200.engine import DeviceGrid
    dev, x0 = bench.build_device()
    g = DeviceGrid(dev.params, dev.idx, dev.material, "mixed", 8)
    x = g.pack(x0)
    rng = np.random.default_rng(4)
    p = g.pack(x0 + 0.1 * rng.standard_normal(x0.shape[0]))
    B = (0.0, 0.0, 0.5)
    want = g.jvp(x, p, 0.1, "krylov", B=B).clone()
    g.set_limits(wait_ns=1)
    with pytest.raises(L.TDGLError) as e:
        g.jvp(x, p, 0.1, "krylov", B=B)
    assert e.value.status == L.TDGL_ETIMEOUT
    g.set_limits()
    got = g.jvp(x, p, 0.1, "krylov", B=B)
    assert torch.equal(got, want)


def test_standalone_kernels_after_a_wait_runs_out():
    """Standalone launches (the Arnoldi-step probe, outside any graph) on a
    fresh context whose wait limit runs out: the staged stencil records the
    timeout, and the projections that follow only record the status (outside
    the graph there are no conditional nodes to stop).  The context then
    steps exactly as a fresh one."""
    from nanowire_tdgl_b200 import _lib as L
    from nanowire_tdgl_b200.engine import stream_handle
    mk, x0, opts, fld = _setup("mixed")
    ref = mk()
    rc, want = _run(ref, x0, opts, fld)
    assert rc == L.TDGL_OK
    g = mk()
    g.set_limits(wait_ns=1)
    # the graph's Arnoldi-step kernels at basis index 2: orthogonalisation,
    # polynomial steps, product, projections
    L.check(g.lib.tdgl_arnoldi_probe(g.handle, 2, 1, 0, stream_handle()), "tdgl_arnoldi_probe")
    torch.cuda.synchronize()
    g.set_limits()
    rc, got = _run(g, x0, opts, fld)
    assert rc == L.TDGL_OK
    assert torch.equal(got, want)
