"""Host-side permutation between the reference state layout and the device
layout (component arrays, nodes i fastest), for tests."""

import numpy as np


def dims(p):
    nx, ny = p.Nx - 1, p.Ny - 1
    nz = p.Nz - 1 if p.Nz > 1 else 1
    return nx, ny, nz


def perm_dev_to_ref(p):
    """r[d]: reference interior index of device node d."""
    nx, ny, nz = dims(p)
    ref = np.arange(nx * ny * nz).reshape(nx, ny, nz)   # ref[i, j, k]
    return ref.transpose(2, 1, 0).ravel()                # device order: i fastest


def to_device(X, p, npad):
    n = p.n_interior
    nb = p.n_state // n
    r = perm_dev_to_ref(p)
    out = np.zeros((nb + 1) * npad)
    out[:n] = X[:n].real[r]
    out[npad:npad + n] = X[:n].imag[r]
    for a in range(1, nb):
        out[(a + 1) * npad:(a + 1) * npad + n] = X[a * n:(a + 1) * n].real[r]
    return out


def to_reference(x, p, npad):
    n = p.n_interior
    nb = p.n_state // n
    r = perm_dev_to_ref(p)
    out = np.zeros(p.n_state, dtype=np.complex128)
    psi = np.empty(n, dtype=np.complex128)
    psi[r] = x[:n] + 1j * x[npad:npad + n]
    out[:n] = psi
    for a in range(1, nb):
        v = np.empty(n)
        v[r] = x[(a + 1) * npad:(a + 1) * npad + n]
        out[a * n:(a + 1) * n] = v
    return out
