"""The tangent-linear stencil of the analytic-product Krylov solves, launched
alone through ``tdgl_jvp(..., TDGL_JVP_KRYLOV)``: ap = p - dt/2 J(x) p as the
step graph computes it (linearisation and direction staged on the full grid,
the product kernel, interior entries back).

* FP64 contexts (kg_arn_apply<double>) against the FP64 analytic product
  (tdgl_jvp ANALYTIC, the stencil on the device layout): 1e-12 relative —
  the staging and the boundary procedure of the full-grid copies.
* Mixed contexts (FP32 vectors; the TMA-staged kernel on 3-D grids) against
  the FP64 product: 2e-6 relative to max |ap| (FP32 rounding of the inputs and
  the stencil).
* The TMA-staged kernel (one and two nodes per thread, TDGL_TL_NX) against
  the FP32 kernel that reads global memory (TDGL_TMA=0): 1e-6 relative (same
  arithmetic, contraction order may differ).
* Holes through the x, y and z faces (ghost nodes with hole links, whose face
  copies read the link flags): the same bounds.
* z-chunking of the TMA-staged kernel (TDGL_TL_CHUNKS): bit-identical outputs
  for every chunk count.
* The 128x128x32 bench device (4 x 16 tiles per plane, the hole): FP32 against
  FP64 at 2e-6.

The operator is the Jacobian of eval_f (src/tdgl3d/physics/rhs.py:147-239),
which the FP64 product matches to 1e-8 against central differences of the
oracle (test_gpu_parity.py).
"""

import numpy as np
import pytest
import torch

from conftest import device_from_fixture, golden, golden_names

pytestmark = pytest.mark.gpu

CASES = golden_names("case_")
DT = 0.1


def _state_and_direction(dev, seed=3):
    rng = np.random.default_rng(seed)
    p = dev.params
    n = p.n_interior
    X = np.zeros(p.n_state, dtype=np.complex128)
    X[:n] = 1.0 + 0.2 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    X[n:] = 0.3 * rng.standard_normal(p.n_state - n)
    P = np.zeros(p.n_state, dtype=np.complex128)
    P[:n] = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    P[n:] = rng.standard_normal(p.n_state - n)
    return X, P


def _products(dev, X, P, B, precision="mixed", env=None, monkeypatch=None):
    from nanowire_tdgl_b200.engine import DeviceGrid
    if env:
        for k, v in env.items():
            monkeypatch.setenv(k, v)
    g64 = DeviceGrid(dev.params, dev.idx, dev.material, "fp64", 8)
    g = DeviceGrid(dev.params, dev.idx, dev.material, precision, 8)
    x, p = g64.pack(X), g64.pack(P)
    want = g64.unpack(g64.jvp(x, p, DT, "analytic", B=B)).cpu().numpy()
    got = g.unpack(g.jvp(x, p, DT, "krylov", B=B)).cpu().numpy()
    torch.cuda.synchronize()
    if env:
        for k in env:
            monkeypatch.delenv(k)
    return got, want


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("name", CASES)
def test_fp64_context_product_matches_analytic(name):
    d = golden(name)
    dev = device_from_fixture(d)
    X, P = _state_and_direction(dev)
    got, want = _products(dev, X, P, tuple(d["B"]), "fp64")
    assert _rel(got, want) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_mixed_context_product_matches_fp64(name):
    d = golden(name)
    dev = device_from_fixture(d)
    X, P = _state_and_direction(dev)
    got, want = _products(dev, X, P, tuple(d["B"]), "mixed")
    assert _rel(got, want) < 2e-6


def _tiled_device(tb, periodic=(False, False, False)):
    px, py, pz = periodic
    p = tb.SimulationParameters(Nx=70, Ny=20, Nz=12, hx=0.5, hy=0.5, hz=0.5, kappa=2.0,
                                periodic_x=px, periodic_y=py, periodic_z=pz)
    dev = tb.Device(p, applied_field=tb.AppliedField(Bz=0.4, By=0.1, t_on_fraction=1.0))
    dev.add_hole([(10.0, 3.0), (14.0, 3.0), (14.0, 6.0), (10.0, 6.0)], z_range=(2, 7))
    return dev


@pytest.mark.parametrize("nx", ["1", "2"])
@pytest.mark.parametrize("periodic", [(False, False, False), (True, True, True)])
def test_tma_kernel_against_global_memory_kernel(monkeypatch, periodic, nx):
    import nanowire_tdgl_b200 as tb
    dev = _tiled_device(tb, periodic)
    X, P = _state_and_direction(dev, 5)
    B = (0.05, 0.1, 0.4)
    tma, want = _products(dev, X, P, B, "mixed", {"TDGL_TL_NX": nx}, monkeypatch)
    plain, _ = _products(dev, X, P, B, "mixed", {"TDGL_TMA": "0"}, monkeypatch)
    assert _rel(tma, want) < 2e-6
    assert _rel(plain, want) < 2e-6
    assert _rel(tma, plain) < 1e-6


def _face_hole_device(tb, periodic):
    px, py, pz = periodic
    p = tb.SimulationParameters(Nx=70, Ny=20, Nz=12, hx=0.5, hy=0.5, hz=0.5, kappa=2.0,
                                periodic_x=px, periodic_y=py, periodic_z=pz)
    dev = tb.Device(p, applied_field=tb.AppliedField(Bz=0.4, By=0.1, t_on_fraction=1.0))
    dev.add_hole([(0.0, 3.0), (4.0, 3.0), (4.0, 6.0), (0.0, 6.0)])              # through the x = 0 face
    dev.add_hole([(20.0, 7.0), (26.0, 7.0), (26.0, 10.0), (20.0, 10.0)], z_range=(0, 5))   # y = Ny and z = 0 faces
    return dev


def _ghosts_with_hole_links(dev):
    """Ghost nodes (one past a face, inside the other two axes' interior range)
    that carry hole links: the face copies of the nodes next to them keep those
    links at zero."""
    p = dev.params
    Nx, Ny, Nz = p.Nx, p.Ny, p.Nz
    hit = np.zeros((Nz + 1) * (Ny + 1) * (Nx + 1), bool)
    for a in "xyz":
        hit[np.asarray(getattr(dev.idx, f"hole_{a}_bc_mask"), dtype=np.int64)] = True
    hit = hit.reshape(Nz + 1, Ny + 1, Nx + 1)
    ghost = np.zeros_like(hit)
    ghost[1:Nz, 1:Ny, [0, Nx]] = True
    ghost[1:Nz, [0, Ny], 1:Nx] = True
    ghost[[0, Nz], 1:Ny, 1:Nx] = True
    return int((hit & ghost).sum())


@pytest.mark.parametrize("nx", ["1", "2"])
@pytest.mark.parametrize("periodic", [(False, False, False), (True, True, True)])
def test_tma_kernel_with_holes_through_faces(monkeypatch, periodic, nx):
    """Holes that reach the x, y and z faces: the face copies of the output
    read the ghosts' link flags (the nodes flagged NF_GHOSTLF)."""
    import nanowire_tdgl_b200 as tb
    dev = _face_hole_device(tb, periodic)
    assert _ghosts_with_hole_links(dev) > 0
    X, P = _state_and_direction(dev, 9)
    B = (0.05, 0.1, 0.4)
    tma, want = _products(dev, X, P, B, "mixed", {"TDGL_TL_NX": nx}, monkeypatch)
    plain, _ = _products(dev, X, P, B, "mixed", {"TDGL_TMA": "0"}, monkeypatch)
    assert _rel(tma, want) < 2e-6
    assert _rel(tma, plain) < 1e-6


@pytest.mark.parametrize("nx", ["1", "2"])
def test_tma_chunks_are_bit_identical(monkeypatch, nx):
    import nanowire_tdgl_b200 as tb
    dev = _tiled_device(tb)
    X, P = _state_and_direction(dev, 6)
    B = (0.0, 0.0, 0.4)
    outs = [_products(dev, X, P, B, "mixed", {"TDGL_TL_CHUNKS": str(c), "TDGL_TL_NX": nx}, monkeypatch)[0]
            for c in (1, 2, 4, 11)]
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])


def test_product_at_headline_size():
    import bench
    dev, x0 = bench.build_device()
    X, P = _state_and_direction(dev, 8)
    got, want = _products(dev, X, P, (0.0, 0.0, bench.WORKLOAD["Bz"]), "mixed")
    assert _rel(got, want) < 2e-6
