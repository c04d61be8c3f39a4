"""Post-processing of solutions: vortex counting and steady-state detection
(src/tdgl3d/analysis/vortex_counting.py, convergence.py), same names,
arguments and return values.

The per-plaquette phase winding of a state (every slice at once) and the
masked means of |psi|^2 and |J_s| that the steady-state check compares run as
CUDA kernels (``tdgl_plaquette_winding``, ``tdgl_convergence_means``); the
remaining logic (thresholds, scan order, windows) is the reference's, on the
host.  ``count_hole_flux_quanta``, ``find_vortex_cores`` and
``count_vortices_polygon`` are host logic on the solution's observables.

Two reference behaviours are kept on purpose, so that answers match it:
``compute_convergence_metrics`` never compares the supercurrent (the
reference's call into the current-density routine raises and it records the
message under ``current_error``; ``include_current=True`` computes the
intended current metrics on the device instead), and
``count_vortices_polygon`` reads the full-grid vector reshaped as
(Nx+1, Ny+1, Nz+1) in C order, as the reference does.
"""

from __future__ import annotations

import numpy as np
import torch

from .engine import grid_for

# what the reference records when its supercurrent comparison fails (it always does)
_CURRENT_ERROR = "eval_supercurrent_density() got an unexpected keyword argument 'step'"


def _material(device):
    return getattr(device, "material", None) if device is not None else None


def _grid(solution, device=None):
    return grid_for(solution.params, solution.idx, _material(device), "fp64")


def _packed(g, solution, step: int) -> torch.Tensor:
    return g.pack(np.ascontiguousarray(np.asarray(solution.states)[:, step]))


def plaquette_windings(solution, step: int = -1, mask_threshold: float = 0.02, device=None) -> np.ndarray:
    """Winding numbers of every plaquette of every interior slice at a saved
    step: shape (max(Nz-1, 1), Nx-2, Ny-2), index [k, i, j] for the plaquette
    with corners at interior nodes (i, j) .. (i+1, j+1) of slice k; NaN where a
    corner's |psi|^2 is below ``mask_threshold``.  (No reference counterpart:
    the reference scans one slice in a Python loop.)"""
    g = _grid(solution, device)
    return g.plaquette_winding(_packed(g, solution, step), mask_threshold).cpu().numpy()


def count_vortices_plaquette(solution, device, slice_z: int = 0, step: int = -1, winding_threshold: float = 0.8,
                             mask_threshold: float = 0.02):
    """Vortices of one slice by plaquette phase winding
    (vortex_counting.py:14-139): (count, positions (n, 2) at plaquette centres
    (i + 0.5, j + 0.5), winding numbers (n,)), in the reference's i-major
    scan order."""
    w = plaquette_windings(solution, step, mask_threshold, device)[slice_z]
    sel = np.abs(np.nan_to_num(w, nan=0.0)) > winding_threshold
    ii, jj = np.nonzero(sel)
    if ii.size == 0:
        return 0, np.empty((0, 2)), np.empty(0)
    return int(ii.size), np.column_stack([ii + 0.5, jj + 0.5]).astype(float), w[sel]


def count_vortices_polygon(solution, device, polygon_points, slice_z: int = 0, step: int = -1) -> float:
    """Phase winding along a closed polygon of full-grid points, in flux
    quanta (vortex_counting.py:142-274)."""
    params, idx = solution.params, solution.idx
    n = params.n_interior
    full = np.zeros(params.dim_x, dtype=np.complex128)
    full[np.asarray(idx.interior_to_full)] = np.asarray(solution.states)[:n, step]
    nx, ny = params.Nx + 1, params.Ny + 1
    if params.Nz == 1:
        sl = full.reshape(nx, ny)
    else:
        sl = full.reshape(nx, ny, params.Nz + 1)[:, :, slice_z + 1]
    poly = np.array(polygon_points)
    if not np.allclose(poly[0], poly[-1]):
        poly = np.vstack([poly, poly[0:1]])
    total = 0.0
    for a, b in zip(poly[:-1], poly[1:]):
        i1, j1 = int(np.clip(a[0], 0, nx - 1)), int(np.clip(a[1], 0, ny - 1))
        i2, j2 = int(np.clip(b[0], 0, nx - 1)), int(np.clip(b[1], 0, ny - 1))
        d = np.angle(sl[i2, j2]) - np.angle(sl[i1, j1])
        total += np.arctan2(np.sin(d), np.cos(d))
    return float(total / (2.0 * np.pi))


def count_hole_flux_quanta(solution, device, hole_bounds, slice_z: int = 0, step: int = -1) -> float:
    """Magnetic flux through a rectangle of interior nodes in flux quanta
    (vortex_counting.py:277-370): sum of Bz (with boundary conditions) times
    hx hy over 2 pi."""
    params = solution.params
    _, _, Bz = solution.bfield(step=step, full_interior=True)
    nx, ny, nz = params.Nx - 1, params.Ny - 1, max(params.Nz - 1, 1)
    bz = np.asarray(Bz).reshape(nx, ny, nz)[:, :, slice_z]
    x_min, x_max, y_min, y_max = hole_bounds
    i0, i1 = max(0, int(x_min)), min(nx, int(x_max))
    j0, j1 = max(0, int(y_min)), min(ny, int(y_max))
    return float(np.sum(bz[i0:i1, j0:j1]) * params.hx * params.hy / (2.0 * np.pi))


def find_vortex_cores(solution, device, slice_z: int = 0, step: int = -1, threshold: float = 0.1,
                      separation: int = 2) -> np.ndarray:
    """Local minima of |psi|^2 below ``threshold`` in one slice
    (vortex_counting.py:373-430), as float (i, j) indices."""
    from scipy.ndimage import minimum_filter
    params = solution.params
    nx, ny, nz = params.Nx - 1, params.Ny - 1, max(params.Nz - 1, 1)
    p2 = (np.abs(np.asarray(solution.states)[:params.n_interior, step]) ** 2).reshape(nx, ny, nz)[:, :, slice_z]
    is_min = (p2 == minimum_filter(p2, size=separation)) & (p2 < threshold)
    return np.argwhere(is_min).astype(float)


class _Means:
    """Per-step [mean |psi|^2, mean |J_s|] of a solution, each saved state
    packed and reduced on the device once."""

    def __init__(self, solution, device):
        self.solution = solution
        self.g = _grid(solution, device)
        mat = _material(device)
        self.sc = (torch.as_tensor(np.asarray(mat.interior_sc_mask, dtype=np.float64), device=self.g.device)
                   if mat is not None else None)
        self.cache = {}

    def __call__(self, step: int):
        if step not in self.cache:
            out = self.g.convergence_means(_packed(self.g, self.solution, step), self.sc).cpu().numpy()
            self.cache[step] = (float(out[0]), float(out[1]))
        return self.cache[step]


def _rel(cur: float, past: float) -> float:
    return abs(cur - past) / cur if cur > 1e-10 else float("inf")


def _metrics(means: _Means, n_steps: int, step: int, window_size: int, with_device: bool,
             include_current: bool) -> dict:
    if step < 0:
        step = n_steps + step
    past = max(0, step - window_size)
    (p_cur, j_cur), (p_past, j_past) = means(step), means(past)
    m = {"psi2_mean_current": p_cur, "psi2_mean_past": p_past, "psi2_rel_change": _rel(p_cur, p_past)}
    if with_device:
        if include_current:
            m.update(current_mean_current=j_cur, current_mean_past=j_past, current_rel_change=_rel(j_cur, j_past))
        else:
            m["current_error"] = _CURRENT_ERROR
    return m


def compute_convergence_metrics(solution, device=None, step: int = -1, window_size: int = 10,
                                include_current: bool = False) -> dict:
    """Relative change of mean |psi|^2 (over superconducting nodes when the
    device has a material map) between saved step ``step`` and
    ``step - window_size`` (convergence.py:14-117).  With a device the
    reference's supercurrent comparison fails and it records ``current_error``;
    ``include_current=True`` adds the mean |J_s| metrics instead."""
    return _metrics(_Means(solution, device), solution.n_steps, step, window_size, device is not None,
                    include_current)


def check_steady_state(solution, device=None, window_size: int = 10, psi_threshold: float = 1e-4,
                       current_threshold: float = 1e-4, start_step: int = 20, include_current: bool = False):
    """First saved step from ``start_step`` on whose metrics are below the
    thresholds (convergence.py:120-197): (is_steady, steady_step or -1, final
    metrics with ``steady_time`` / ``steady_step`` when found)."""
    means = _Means(solution, device)
    n_steps = solution.n_steps
    dev = device is not None

    def metrics(step):
        return _metrics(means, n_steps, step, window_size, dev, include_current)

    if n_steps < start_step + window_size:
        return False, -1, metrics(-1)
    steady = -1
    for step in range(start_step, n_steps):
        m = metrics(step)
        ok = m["psi2_rel_change"] < psi_threshold
        if dev and "current_rel_change" in m:
            ok = ok and m["current_rel_change"] < current_threshold
        if ok:
            steady = step
            break
    final = metrics(-1)
    if steady >= 0:
        final["steady_time"] = float(np.asarray(solution.times)[steady])
        final["steady_step"] = steady
        return True, steady, final
    return False, -1, final
