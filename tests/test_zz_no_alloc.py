"""The allocation-free RHS entry point, tdgl_eval_f_noalloc.

It serves callers that may not allocate device memory when they run; it takes
the grid and material descriptors directly (no context) and keeps all of its
intermediates in one static device array.  Its output must equal the
context-based tdgl_eval_f on the same inputs, call after call: the array keeps
the previous call's contents, so two different states are evaluated in a row
for every geometry.  This file is collected last on purpose.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from conftest import device_from_fixture, golden

pytestmark = pytest.mark.gpu

CASES = ["case_3d_hole_edge", "case_trilayer_hole", "case_2d_hole_triangle", "case_continuous_sc",
         "case_3d_periodic_yz", "case_config1", "case_3d_basic"]
RTOL = 1e-12   # the RHS tolerance of the other GPU parity tests


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-300))


@pytest.mark.parametrize("name", CASES)
def test_noalloc_matches_context_eval_f(name):
    from nanowire_tdgl_b200 import _lib
    from nanowire_tdgl_b200.engine import descriptors, grid_for, stream_handle
    lib = _lib.load()
    d = golden(name)
    dev = device_from_fixture(d)
    B = tuple(float(b) for b in d["B"])
    ctx_grid = grid_for(dev.params, dev.idx, dev.material)
    gd, md, keep = descriptors(dev.params, dev.idx, dev.material)
    states = [d["X_seeded"], d["X_random"] if "X_random" in d else 0.5 * d["X_seeded"]]
    for X in states:                               # two calls in a row on the shared array
        want = ctx_grid.eval_f_ref(X, B)           # existing entry point (tdgl_eval_f)
        x = ctx_grid.ref_tensor(X)
        f = torch.full_like(x, float("nan"))
        rc = lib.tdgl_eval_f_noalloc(C.byref(gd), C.byref(md), C.c_void_p(x.data_ptr()),
                                     C.c_void_p(f.data_ptr()), *B, stream_handle())
        assert rc == _lib.TDGL_OK, lib.tdgl_last_error()
        torch.cuda.synchronize()
        assert _rel(f, want) < RTOL


def _limit_device():
    """33x33x33 cells: 32,768 interior nodes (the entry point's limit), a hole
    through part of the thickness, per-node kappa and fractional sc."""
    import nanowire_tdgl_b200 as tb
    p = tb.SimulationParameters(Nx=33, Ny=33, Nz=33, hx=0.5, hy=0.5, hz=0.5, kappa=2.0)
    dev = tb.Device(p, applied_field=tb.AppliedField(Bx=0.1, Bz=0.5, t_on_fraction=1.0))
    dev.add_hole([(4.0, 4.0), (8.0, 4.0), (8.0, 7.5), (4.0, 7.5)], z_range=(3, 20))
    m = dev.material
    rng = np.random.default_rng(21)
    kappa = m.kappa * (1.0 + 0.3 * rng.random(m.kappa.shape))
    sc = m.interior_sc_mask * (0.5 + 0.5 * rng.random(m.interior_sc_mask.shape))
    dev._material = tb.MaterialMap(kappa=kappa, sc_mask=m.sc_mask.copy(), interior_sc_mask=sc)
    assert p.n_interior == 32768
    return dev


def test_noalloc_at_its_limit_after_a_smaller_grid():
    """At the maximum size, after a smaller geometry has filled the array:
    two calls in a row (different states) against tdgl_eval_f."""
    from nanowire_tdgl_b200 import _lib
    from nanowire_tdgl_b200.engine import descriptors, grid_for, stream_handle
    lib = _lib.load()
    small = device_from_fixture(golden("case_3d_hole"))
    big = _limit_device()
    rng = np.random.default_rng(22)
    for dev, calls in ((small, 1), (big, 2)):
        ctx_grid = grid_for(dev.params, dev.idx, dev.material)
        gd, md, keep = descriptors(dev.params, dev.idx, dev.material)
        n = dev.params.n_interior
        for _ in range(calls):
            X = np.zeros(dev.params.n_state, dtype=np.complex128)
            X[:n] = 1.0 + 0.3 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
            X[n:] = 0.2 * rng.standard_normal(dev.params.n_state - n)
            B = (0.1, 0.0, 0.5)
            want = ctx_grid.eval_f_ref(X, B)
            x = ctx_grid.ref_tensor(X)
            f = torch.full_like(x, float("nan"))
            rc = lib.tdgl_eval_f_noalloc(C.byref(gd), C.byref(md), C.c_void_p(x.data_ptr()),
                                         C.c_void_p(f.data_ptr()), *B, stream_handle())
            assert rc == _lib.TDGL_OK, lib.tdgl_last_error()
            torch.cuda.synchronize()
            assert _rel(f, want) < RTOL


def test_noalloc_rejects_grids_beyond_its_limit():
    from nanowire_tdgl_b200 import _lib
    lib = _lib.load()
    gd = _lib.GridDesc(200, 200, 2, 0, 0, 0, 0.5, 0.5, 0.5, 2.0)     # 39601 interior nodes > 32768
    x = torch.zeros(2 * 3 * 199 * 199, dtype=torch.float64, device="cuda")
    rc = lib.tdgl_eval_f_noalloc(C.byref(gd), None, C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()),
                                 0.0, 0.0, 0.0, None)
    assert rc == _lib.TDGL_EINVAL
    assert b"at most 32768 interior nodes" in lib.tdgl_last_error()
