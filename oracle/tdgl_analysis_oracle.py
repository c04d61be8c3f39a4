"""CPU oracle for the analysis kernels — TEST INFRASTRUCTURE ONLY.

Plain-numpy restatement of the plaquette phase winding
(src/tdgl3d/analysis/vortex_counting.py:14-139, _wrap_phase :433-435) and of
the masked means that compute_convergence_metrics compares
(src/tdgl3d/analysis/convergence.py:14-117).  Imported only by ``tests/``;
pinned against ``tests/golden/analysis.npz``, which the reference itself
produced (``tests/golden/make_analysis_golden.py``).
"""

from __future__ import annotations

import numpy as np


def plaquette_windings(psi_ref: np.ndarray, Nx: int, Ny: int, Nz: int, mask_threshold: float) -> np.ndarray:
    """Winding number of every plaquette of every interior slice,
    shape (slices, Nx-2, Ny-2), NaN where a corner's |psi|^2 is below the
    threshold.  psi_ref in reference interior order (k fastest)."""
    nx, ny, nz = Nx - 1, Ny - 1, max(Nz - 1, 1)
    psi = np.asarray(psi_ref).reshape(nx, ny, nz).transpose(2, 0, 1)      # [k, i, j]
    p2 = np.abs(psi) ** 2
    ph = np.angle(psi)
    corners = [(0, 0), (1, 0), (1, 1), (0, 1)]
    sl = [(slice(None), slice(di, nx - 1 + di), slice(dj, ny - 1 + dj)) for di, dj in corners]
    masked = np.zeros((nz, nx - 1, ny - 1), dtype=bool)
    for s in sl:
        masked |= p2[s] < mask_threshold
    w = np.zeros((nz, nx - 1, ny - 1))
    for c in range(4):
        d = ph[sl[(c + 1) % 4]] - ph[sl[c]]
        w = w + np.arctan2(np.sin(d), np.cos(d))
    w = w / (2.0 * np.pi)
    w[masked] = np.nan
    return w


def count_vortices_plaquette(psi_ref, Nx, Ny, Nz, slice_z=0, winding_threshold=0.8, mask_threshold=0.02):
    """(n, positions (n, 2), windings (n,)) for one slice, i-major order."""
    w = plaquette_windings(psi_ref, Nx, Ny, Nz, mask_threshold)[slice_z]
    sel = np.abs(np.nan_to_num(w, nan=0.0)) > winding_threshold
    ii, jj = np.nonzero(sel)
    pos = np.column_stack([ii + 0.5, jj + 0.5]) if ii.size else np.empty((0, 2))
    return int(ii.size), pos, w[sel] if ii.size else np.empty(0)


def masked_means(psi_ref, J, sc=None):
    """Mean |psi|^2 and mean |J_s| over nodes with sc > 0 (all without sc);
    J = (Jx, Jy, Jz or None) in reference order."""
    p2 = np.abs(np.asarray(psi_ref)) ** 2
    jx, jy, jz = J
    jm = np.sqrt(jx ** 2 + jy ** 2 + (jz ** 2 if jz is not None else 0))
    if sc is not None:
        m = np.asarray(sc) > 0
        return float(np.mean(p2[m])), float(np.mean(jm[m]))
    return float(np.mean(p2)), float(np.mean(jm))
