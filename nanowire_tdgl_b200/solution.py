"""Result container with the observables of src/tdgl3d/core/solution.py:20-217.

|psi|^2, B (boundary-extended links, applied field at the saved time) and the
supercurrent J_s (zero-extended state, no boundary conditions) are evaluated
by the device observables kernel.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from .engine import grid_for


@dataclass
class Solution:
    times: np.ndarray
    states: np.ndarray
    params: object
    idx: object
    device: Optional[object] = None
    metadata: Optional[dict] = None

    @property
    def n_steps(self) -> int:
        return self.states.shape[1]

    def psi(self, step: int = -1):
        return self.states[: self.params.n_interior, step]

    def phi_x(self, step: int = -1):
        n = self.params.n_interior
        return self.states[n: 2 * n, step]

    def phi_y(self, step: int = -1):
        n = self.params.n_interior
        return self.states[2 * n: 3 * n, step]

    def phi_z(self, step: int = -1):
        if not self.params.is_3d:
            raise AttributeError("No phi_z for 2-D simulations.")
        n = self.params.n_interior
        return self.states[3 * n: 4 * n, step]

    def phase(self, step: int = -1, mask_threshold: float = 0.02):
        psi = np.asarray(self.psi(step))
        ph = np.angle(psi).astype(np.float64)
        ph[np.abs(psi) ** 2 < mask_threshold] = np.nan
        return ph

    # -- device observables -------------------------------------------------
    def _observe(self, step: int, with_field: bool) -> dict:
        material = getattr(self.device, "material", None) if self.device is not None else None
        g = grid_for(self.params, self.idx, material, "fp64")
        x = g.pack(np.asarray(self.states[:, step]))
        B = (0.0, 0.0, 0.0)
        if with_field and self.device is not None and getattr(self.device, "applied_field", None) is not None:
            t = float(self.times[step])
            B = self.device.applied_field.evaluate(t, float(self.times[-1]))
        out = g.observables(x, B)
        return {k: v.cpu().numpy() for k, v in out.items()}

    def psi_squared(self, step: int = -1):
        return self._observe(step, False)["psi2"]

    def bfield(self, step: int = -1, full_interior: bool = True):
        """B = curl(phi) at interior nodes after the boundary conditions with
        the applied field at this step's time (solution.py:94-158).  With
        ``full_interior=False`` only the inner subset ``idx.bfield_interior``
        is returned (bfield.py:81-151), taken from the same device values:
        away from the boundary the two definitions coincide."""
        o = self._observe(step, True)
        Bx, By, Bz = o["Bx"], o["By"], o["Bz"]
        if full_interior:
            return Bx, By, Bz
        return self._inner_bfield(step)

    def _inner_bfield(self, step: int):
        # bfield.py:81-151 applies offsets 1, Nx-1 and (Nx-1)(Ny-1) to flat
        # state indices; the same gathers are done here on the device
        p = self.params
        n = p.n_interior
        s = torch.as_tensor(np.asarray(self.states[:, step]), device="cuda").real
        m = torch.as_tensor(np.asarray(self.idx.bfield_interior), device="cuda", dtype=torch.long)
        mj, mk = p.Nx - 1, (p.Nx - 1) * (p.Ny - 1)
        fx, fy = s[n:2 * n], s[2 * n:3 * n]
        Bz = (fx[m] - fx[m + mj] - fy[m] + fy[m + 1]) * (1.0 / (p.hx * p.hy))
        if p.is_3d:
            fz = s[3 * n:4 * n]
            Bx = (fy[m] - fy[m + mk] - fz[m] + fz[m + mj]) * (1.0 / (p.hy * p.hz))
            By = (fz[m] - fz[m + 1] - fx[m] + fx[m + mk]) * (1.0 / (p.hz * p.hx))
        else:
            Bx = torch.zeros_like(Bz)
            By = torch.zeros_like(Bz)
        return Bx.cpu().numpy(), By.cpu().numpy(), Bz.cpu().numpy()

    def supercurrent_density(self, step: int = -1):
        o = self._observe(step, False)
        return o["Jx"], o["Jy"], o["Jz"]

    def normal_current_density(self, step: int = -1):
        return None   # the reference does not store mu either (solution.py:219-247)

    def current_density(self, step: int = -1):
        return self.supercurrent_density(step)

    def current_magnitude(self, step: int = -1, dataset: Optional[str] = None):
        Jx, Jy, Jz = self.supercurrent_density(step)
        return np.sqrt(Jx ** 2 + Jy ** 2 + Jz ** 2)

    def _reshape_interior(self, arr, slice_z: int = 0):
        p = self.params
        if p.is_3d:
            return np.asarray(arr).reshape(p.Nx - 1, p.Ny - 1, max(p.Nz - 1, 1))[:, :, slice_z]
        return np.asarray(arr).reshape(p.Nx - 1, p.Ny - 1)

    def psi_squared_2d(self, step: int = -1, slice_z: int = 0):
        return np.abs(self._reshape_interior(self.psi(step), slice_z)) ** 2

    def count_vortices(self, device, slice_z: int = 0, step: int = -1, method: str = "plaquette", **kwargs):
        """Vortices of one slice by ``method`` (src/tdgl3d/core/solution.py:302-354):
        "plaquette" (``count_vortices_plaquette``: count, positions, windings),
        "polygon" (``count_vortices_polygon``, needs ``polygon_points``) or
        "cores" (``find_vortex_cores``); ValueError for anything else."""
        from . import analysis
        if method == "plaquette":
            return analysis.count_vortices_plaquette(self, device, slice_z, step, **kwargs)
        if method == "polygon":
            if "polygon_points" not in kwargs:
                raise ValueError("polygon method requires polygon_points argument")
            return analysis.count_vortices_polygon(self, device, kwargs["polygon_points"], slice_z, step)
        if method == "cores":
            return analysis.find_vortex_cores(self, device, slice_z, step, **kwargs)
        raise ValueError(f"Unknown method: {method}")

    def check_steady_state(self, device=None, window_size: int = 10, psi_threshold: float = 1e-4,
                           current_threshold: float = 1e-4, start_step: int = 20):
        """``check_steady_state`` on this solution (src/tdgl3d/core/solution.py:356-396)."""
        from . import analysis
        return analysis.check_steady_state(self, device, window_size, psi_threshold, current_threshold, start_step)

    def save(self, filename: str) -> None:
        """HDF5 file in the layout of src/tdgl3d/core/solution.py:400-461
        (times, states, parameters, grid indices, metadata; needs h5py)."""
        from .hdf5 import save_full
        save_full(self, filename)

    @staticmethod
    def load(filename: str) -> "Solution":
        """A ``save`` file (src/tdgl3d/core/solution.py:463-549); the device
        is not stored, so ``device`` is None."""
        from .hdf5 import load_full
        return load_full(filename)
