"""The device stencil code (tdgl_stencil.cuh + tdgl_geometry.h), compiled for
the host, against the oracle and the reference's golden RHS values.

This checks the kernels' index arithmetic, boundary rules, hole/material
flags and the analytic Jacobian product on the CPU; the GPU tests repeat the
comparison through the C ABI on the device."""

import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, device_from_fixture, golden, golden_names
from layout import to_device, to_reference

from nanowire_tdgl_b200.engine import descriptors
from oracle import tdgl_oracle as orc

CASES = golden_names("case_")


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("hoststencil") / "stencil_host.so"
    src = os.path.join(ROOT, "tests", "stencil_host.cpp")
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "nanowire_tdgl_b200", "csrc"), "-o", str(out), src], check=True)
    lib = C.CDLL(str(out))
    P = C.c_void_p
    lib.host_layout.argtypes = [P, P, P, P]
    lib.host_rhs.argtypes = [P, P, P, P, C.c_double, C.c_double, C.c_double]
    lib.host_jvp.argtypes = [P, P, P, P, P, C.c_double, C.c_double, C.c_double, C.c_int]
    lib.host_nflags.argtypes = [P, P, P]
    return lib


def _setup(lib, dev):
    g, md, keep = descriptors(dev.params, dev.idx, dev.material)
    n, npad, nc = C.c_int64(), C.c_int64(), C.c_int64()
    assert lib.host_layout(C.byref(g), C.byref(n), C.byref(npad), C.byref(nc)) == 0
    return g, md, keep, npad.value, nc.value


def _rhs(lib, dev, X, B):
    g, md, keep, npad, nc = _setup(lib, dev)
    x = to_device(X, dev.params, npad)
    f = np.zeros_like(x)
    rc = lib.host_rhs(C.byref(g), C.byref(md), x.ctypes.data, f.ctypes.data, *map(float, B))
    assert rc == 0
    return to_reference(f, dev.params, npad)


def _jvp(lib, dev, X, Pv, B, as_float=0):
    g, md, keep, npad, nc = _setup(lib, dev)
    x = to_device(X, dev.params, npad)
    p = to_device(Pv, dev.params, npad)
    jp = np.zeros_like(x)
    rc = lib.host_jvp(C.byref(g), C.byref(md), x.ctypes.data, p.ctypes.data, jp.ctypes.data, *map(float, B),
                      as_float)
    assert rc == 0
    return to_reference(jp, dev.params, npad)


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("name", CASES)
def test_host_stencil_rhs_matches_reference(host_lib, name):
    d = golden(name)
    dev = device_from_fixture(d)
    F = _rhs(host_lib, dev, d["X_seeded"], d["B"])
    assert _rel(F, d["F_seeded"]) < 1e-12
    if "X_random" in d:
        F = _rhs(host_lib, dev, d["X_random"], d["B"])
        assert _rel(F, d["F_random"]) < 1e-12
        F0 = _rhs(host_lib, dev, d["X_random"], (0.0, 0.0, 0.0))
        assert _rel(F0, d["F_random_b0"]) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_host_stencil_jvp_matches_central_difference(host_lib, name):
    d = golden(name)
    dev = device_from_fixture(d)
    g = orc.make_grid(dev.params, dev.idx, dev.material)
    X = d.get("X_random", d["X_seeded"])
    rng = np.random.default_rng(5)
    n = dev.params.n_interior
    P = rng.standard_normal(dev.params.n_state) + 0j
    P[:n] += 1j * rng.standard_normal(n)
    h = 1e-5
    fd = (orc.eval_f(X + h * P, g, *d["B"]) - orc.eval_f(X - h * P, g, *d["B"])) / (2 * h)
    jp = _jvp(host_lib, dev, X, P, d["B"])
    assert _rel(jp, fd) < 1e-7
    jpf = _jvp(host_lib, dev, X, P, d["B"], as_float=1)
    assert _rel(jpf, fd) < 1e-5


def test_fast_path_covers_interior(host_lib):
    # config-1 geometry: nodes two or more layers from every face take the fast path
    d = golden("case_config1")
    dev = device_from_fixture(d)
    g, md, keep, npad, nc = _setup(host_lib, dev)
    nf = np.zeros(dev.params.n_interior, dtype=np.uint8)
    assert host_lib.host_nflags(C.byref(g), C.byref(md), nf.ctypes.data) == 0
    slow = (nf & 1).astype(bool).reshape(dev.params.Nz - 1, dev.params.Ny - 1, dev.params.Nx - 1)
    assert not slow[1:-2, 1:-2, 1:-2].any()
    assert slow[0].all() and slow[-2:].all()


@pytest.mark.parametrize("periodic", [(False, False, False), (True, True, True), (True, False, True)])
def test_ghost_link_flags(host_lib, periodic):
    """NF_GHOSTLF (bit 6) marks exactly the face nodes whose face copy lands
    on a ghost node that carries hole links (the copy across x = 1 lands on
    i = 0, or i = Nx when x is periodic; likewise for the other faces), for
    holes that reach the x, y and z faces."""
    import nanowire_tdgl_b200 as tb
    px, py, pz = periodic
    p = tb.SimulationParameters(Nx=30, Ny=20, Nz=12, hx=0.5, hy=0.5, hz=0.5, kappa=2.0,
                                periodic_x=px, periodic_y=py, periodic_z=pz)
    dev = tb.Device(p, applied_field=tb.AppliedField(Bz=0.4, t_on_fraction=1.0))
    dev.add_hole([(0.0, 3.0), (4.0, 3.0), (4.0, 6.0), (0.0, 6.0)])                              # x = 0 face
    dev.add_hole([(8.0, 7.0), (12.0, 7.0), (12.0, 10.0), (8.0, 10.0)], z_range=(0, 5))      # y = Ny, z = 0
    Nx, Ny, Nz = p.Nx, p.Ny, p.Nz
    hit = np.zeros((Nz + 1) * (Ny + 1) * (Nx + 1), bool)
    for a in "xyz":
        hit[np.asarray(getattr(dev.idx, f"hole_{a}_bc_mask"), dtype=np.int64)] = True
    hit = hit.reshape(Nz + 1, Ny + 1, Nx + 1)
    want = np.zeros((Nz - 1, Ny - 1, Nx - 1), bool)            # interior nodes, [k-1, j-1, i-1]
    want[:, :, 0] |= hit[1:Nz, 1:Ny, Nx if px else 0]
    want[:, :, -1] |= hit[1:Nz, 1:Ny, 0 if px else Nx]
    want[:, 0, :] |= hit[1:Nz, Ny if py else 0, 1:Nx]
    want[:, -1, :] |= hit[1:Nz, 0 if py else Ny, 1:Nx]
    want[0, :, :] |= hit[Nz if pz else 0, 1:Ny, 1:Nx]
    want[-1, :, :] |= hit[0 if pz else Nz, 1:Ny, 1:Nx]
    assert want.any()
    g, md, keep, npad, nc = _setup(host_lib, dev)
    nf = np.zeros(p.n_interior, dtype=np.uint8)
    assert host_lib.host_nflags(C.byref(g), C.byref(md), nf.ctypes.data) == 0
    got = (nf & (1 << 6)).astype(bool).reshape(Nz - 1, Ny - 1, Nx - 1)
    assert np.array_equal(got, want)
    assert not got[1:-1, 1:-1, 1:-1].any()
