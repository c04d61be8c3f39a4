"""Device, applied field and state-vector containers (host side).

These mirror the objects a tdgl3d user builds before calling ``solve``:

* ``AppliedField`` / ``build_boundary_field_vectors``
  src/tdgl3d/physics/applied_field.py:14-91
* ``BoundaryVectors``                  src/tdgl3d/physics/rhs.py:32-40
* ``StateVector``                      src/tdgl3d/core/state.py:11-121
* ``Device``                           src/tdgl3d/core/device.py:18-169

The device stepper only needs the three field scalars (Bx, By, Bz) at the
start of each step; the full-grid boundary vectors are still produced for
callers that use the reference's ``eval_f(X, params, idx, u)`` signature.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np
from numpy.typing import NDArray

from .geometry import (GridIndices, MaterialMap, SimulationParameters, Trilayer,
                       build_material_map, construct_indices)


@dataclass
class AppliedField:
    """Applied field schedule (src/tdgl3d/physics/applied_field.py:14-56).

    The field is zero for ``t <= 0`` and for ``t > t_on_fraction * t_stop``;
    with ``ramp`` it grows linearly over ``ramp_fraction * t_stop``.  A
    ``field_func(t, t_stop) -> (Bx, By, Bz)`` overrides the schedule."""

    Bx: float = 0.0
    By: float = 0.0
    Bz: float = 0.0
    t_on_fraction: float = 2.0 / 3.0
    ramp: bool = False
    ramp_fraction: float = 0.5
    field_func: Optional[Callable[[float, float], tuple]] = None

    def evaluate(self, t: float, t_stop: float) -> tuple[float, float, float]:
        if self.field_func is not None:
            return self.field_func(t, t_stop)
        if t <= 0 or t > t_stop * self.t_on_fraction:
            return 0.0, 0.0, 0.0
        scale = 1.0
        if self.ramp:
            t_ramp = t_stop * self.ramp_fraction
            scale = min(t / t_ramp, 1.0) if t_ramp > 0 else 1.0
        return self.Bx * scale, self.By * scale, self.Bz * scale


class BoundaryVectors:
    """Full-grid applied-field vectors for one RHS evaluation
    (src/tdgl3d/physics/rhs.py:32-40)."""

    __slots__ = ("Bx", "By", "Bz")

    def __init__(self, Bx: NDArray, By: NDArray, Bz: NDArray):
        self.Bx, self.By, self.Bz = Bx, By, Bz


def build_boundary_field_vectors(applied_bx, applied_by, applied_bz,
                                 params: SimulationParameters, idx: GridIndices):
    """Place each applied component on the inner nodes of the four faces
    parallel to it (src/tdgl3d/physics/applied_field.py:59-91): Bx on the
    y and z faces, By on the z and x faces, Bz on the x and y faces."""
    N = params.dim_x
    vecs = []
    faces = {
        0: ("y", "z"),
        1: ("z", "x"),
        2: ("x", "y"),
    }
    for comp, val in enumerate((applied_bx, applied_by, applied_bz)):
        v = np.zeros(N, dtype=np.float64)
        if val != 0.0:
            a, b = faces[comp]
            sel = np.concatenate([getattr(idx, f"{a}_face_lo_inner"), getattr(idx, f"{b}_face_lo_inner"),
                                  getattr(idx, f"{a}_face_hi_inner"), getattr(idx, f"{b}_face_hi_inner")])
            np.add.at(v, sel, val)
        vecs.append(v)
    return tuple(vecs)


def field_scalars_from_vectors(u, params: SimulationParameters, idx: GridIndices):
    """Recover (Bx, By, Bz) from reference-style boundary vectors.

    The device kernels take one scalar per component, which is exactly what
    ``build_boundary_field_vectors`` encodes.  Any other per-node layout is
    rejected rather than silently approximated."""
    out = []
    faces = {0: ("y", "z"), 1: ("z", "x"), 2: ("x", "y")}
    for comp, name in enumerate(("Bx", "By", "Bz")):
        vec = np.asarray(getattr(u, name), dtype=np.float64)
        if vec.shape != (params.dim_x,):
            raise ValueError(f"u.{name} must have shape ({params.dim_x},)")
        a, b = faces[comp]
        sel = np.concatenate([getattr(idx, f"{a}_face_lo_inner"), getattr(idx, f"{b}_face_lo_inner"),
                              getattr(idx, f"{a}_face_hi_inner"), getattr(idx, f"{b}_face_hi_inner")])
        val = float(vec[sel[0]]) if sel.size else 0.0
        expect = np.zeros_like(vec)
        if val != 0.0:
            np.add.at(expect, sel, val)
        # Only the face entries are read by the boundary conditions; anything
        # else in the vector is ignored there as well.
        if sel.size and not np.array_equal(vec[sel], expect[sel]):
            raise ValueError(
                f"u.{name} is not a uniform applied field on its boundary faces; "
                "the device RHS takes one scalar per field component")
        out.append(val)
    return tuple(out)


class StateVector:
    """Flat complex state ``[psi, phi_x, phi_y, (phi_z)]`` in interior order
    with named views (src/tdgl3d/core/state.py:11-121)."""

    def __init__(self, data: NDArray, params: SimulationParameters):
        if data.shape != (params.n_state,):
            raise ValueError(
                f"State vector length {data.shape} does not match expected "
                f"({params.n_state},) for grid {params.Nx}×{params.Ny}×{params.Nz}.")
        self._data = np.asarray(data, dtype=np.complex128)
        self._params = params

    @property
    def data(self) -> NDArray[np.complex128]:
        return self._data

    def _block(self, b: int) -> slice:
        n = self._params.n_interior
        return slice(b * n, (b + 1) * n)

    @property
    def psi(self):
        return self._data[self._block(0)]

    @psi.setter
    def psi(self, val):
        self._data[self._block(0)] = val

    @property
    def phi_x(self):
        return self._data[self._block(1)]

    @phi_x.setter
    def phi_x(self, val):
        self._data[self._block(1)] = val

    @property
    def phi_y(self):
        return self._data[self._block(2)]

    @phi_y.setter
    def phi_y(self, val):
        self._data[self._block(2)] = val

    @property
    def phi_z(self):
        if not self._params.is_3d:
            raise AttributeError("phi_z is not available for 2-D simulations (Nz == 1).")
        return self._data[self._block(3)]

    @phi_z.setter
    def phi_z(self, val):
        if not self._params.is_3d:
            raise AttributeError("phi_z is not available for 2-D simulations.")
        self._data[self._block(3)] = val

    def copy(self) -> "StateVector":
        return StateVector(self._data.copy(), self._params)

    @classmethod
    def uniform_superconducting(cls, params: SimulationParameters) -> "StateVector":
        data = np.zeros(params.n_state, dtype=np.complex128)
        data[: params.n_interior] = 1.0
        return cls(data, params)

    @classmethod
    def from_components(cls, psi, phi_x, phi_y, phi_z, params: SimulationParameters) -> "StateVector":
        parts = [psi, phi_x, phi_y]
        if params.is_3d:
            if phi_z is None:
                raise ValueError("phi_z required for 3-D.")
            parts.append(phi_z)
        return cls(np.concatenate([np.ravel(p) for p in parts]).astype(np.complex128), params)

    def __repr__(self) -> str:
        p = self._params
        return (f"StateVector(Nx={p.Nx}, Ny={p.Ny}, Nz={p.Nz}, n_interior={p.n_interior}, "
                f"|ψ|_max={np.max(np.abs(self.psi)):.4f})")


@dataclass
class Device:
    """Parameters + applied field + optional trilayer, with index maps and
    material map built on construction (src/tdgl3d/core/device.py:18-169)."""

    params: SimulationParameters
    applied_field: AppliedField = field(default_factory=AppliedField)
    trilayer: Optional[Trilayer] = None
    _idx: Optional[GridIndices] = field(default=None, repr=False, init=False)
    _material: Optional[MaterialMap] = field(default=None, repr=False, init=False)

    def __post_init__(self) -> None:
        if self.trilayer is not None and self.params.Nz != self.trilayer.Nz:
            object.__setattr__(self.params, "Nz", self.trilayer.Nz)
        self._idx = construct_indices(self.params)
        if self.trilayer is not None:
            self._material = build_material_map(self.params, self.trilayer, self._idx)

    @property
    def idx(self) -> GridIndices:
        if self._idx is None:
            self._idx = construct_indices(self.params)
        return self._idx

    @property
    def material(self) -> Optional[MaterialMap]:
        return self._material

    def initial_state(self) -> StateVector:
        sv = StateVector.uniform_superconducting(self.params)
        if self._material is not None:
            sv.psi[:] *= self._material.interior_sc_mask
        return sv

    def rebuild_indices(self) -> None:
        self._idx = construct_indices(self.params)
        if self.trilayer is not None:
            self._material = build_material_map(self.params, self.trilayer, self._idx)

    def add_hole(self, vertices, z_range: Optional[tuple[int, int]] = None) -> None:
        """Register a polygon hole: hole-boundary links in the index maps and
        sc_mask = 0 inside; a uniform material map is created first when the
        device has none (src/tdgl3d/core/device.py:80-153)."""
        if z_range is None:
            z_range = (0, self.params.Nz)
        self.idx.define_hole_polygon(vertices, z_range, self.params)
        if self._material is None:
            p = self.params
            self._material = MaterialMap(
                kappa=np.full(p.dim_x, p.kappa, dtype=np.float64),
                sc_mask=np.ones(p.dim_x, dtype=np.float64),
                interior_sc_mask=np.ones(p.n_interior, dtype=np.float64))
        self._material.carve_hole_polygon(vertices, z_range, self.params, self.idx)

    def __repr__(self) -> str:
        p = self.params
        f = self.applied_field
        return (f"Device(Nx={p.Nx}, Ny={p.Ny}, Nz={p.Nz}, κ={p.kappa}, "
                f"field=({f.Bx}, {f.By}, {f.Bz}))")
