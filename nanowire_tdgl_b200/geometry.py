"""Grid description, integer index maps, hole rasterisation and material maps.

Host-side set-up for the device stepper.  Everything here is integer or
bit-exact floating-point bookkeeping that runs once per device; none of it is
on the per-step path.  The arrays reproduce, element for element and in the
same order, the index maps that tdgl3d builds, because callers of the
reference read them directly (``idx.interior_to_full``, ``idx.hole_x_bc_mask``
and so on) and because the device flag arrays are derived from them.

Reference interfaces mirrored here (paths inside the tdgl3d project):

* ``SimulationParameters``      src/tdgl3d/core/parameters.py:10-94
* ``GridIndices``/``construct_indices`` src/tdgl3d/mesh/indices.py:62-450
* ``point_in_polygon`` / ``identify_hole_nodes`` / ``identify_boundary_links``
  / ``identify_circular_hole_nodes``  src/tdgl3d/mesh/holes.py:43-311
* ``MaterialMap`` / ``Layer`` / ``Trilayer`` / ``build_material_map``
  src/tdgl3d/core/material.py:26-254
"""

from __future__ import annotations

import copy as _copy
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np
from numpy.typing import NDArray

_EMPTY = lambda: np.array([], dtype=np.intp)  # noqa: E731


# ---------------------------------------------------------------------------
# Parameters
# ---------------------------------------------------------------------------

@dataclass
class SimulationParameters:
    """Grid and physics parameters (same fields, defaults and validation as
    src/tdgl3d/core/parameters.py:10-51).

    ``Nx, Ny, Nz`` count grid *cells*; the full grid has ``(Nx+1)(Ny+1)(Nz+1)``
    nodes and the state lives on the ``(Nx-1)(Ny-1)max(Nz-1,1)`` interior
    nodes.  ``Nz == 1`` selects the quasi-2-D model.
    """

    Nx: int = 10
    Ny: int = 10
    Nz: int = 1
    hx: float = 1.0
    hy: float = 1.0
    hz: float = 1.0
    kappa: float = 5.0
    periodic_x: bool = False
    periodic_y: bool = False
    periodic_z: bool = False

    def __post_init__(self) -> None:
        if self.Nx < 2 or self.Ny < 2:
            raise ValueError("Nx and Ny must each be >= 2.")
        if self.Nz < 1:
            raise ValueError("Nz must be >= 1.")

    @property
    def is_3d(self) -> bool:
        return self.Nz > 1

    @property
    def n_interior(self) -> int:
        return (self.Nx - 1) * (self.Ny - 1) * max(self.Nz - 1, 1)

    @property
    def n_full(self) -> int:
        return (self.Nx + 1) * (self.Ny + 1) * ((self.Nz + 1) if self.is_3d else 1)

    @property
    def n_state(self) -> int:
        return (4 if self.is_3d else 3) * self.n_interior

    @property
    def dim_x(self) -> int:
        return self.n_full

    @property
    def mj(self) -> int:
        return self.Nx + 1

    @property
    def mk(self) -> int:
        return (self.Nx + 1) * (self.Ny + 1)

    def copy(self) -> "SimulationParameters":
        return _copy.deepcopy(self)


# ---------------------------------------------------------------------------
# Index maps
# ---------------------------------------------------------------------------

@dataclass
class GridIndices:
    """Index arrays of the full grid (field names as in
    src/tdgl3d/mesh/indices.py:62-134).  All indices are 0-based full-grid
    linear indices ``m = i + mj*j + mk*k`` unless the name says *interior*."""

    interior_to_full: NDArray[np.intp] = field(default_factory=_EMPTY)
    bfield_interior: NDArray[np.intp] = field(default_factory=_EMPTY)

    x_face_lo: NDArray[np.intp] = field(default_factory=_EMPTY)
    x_first: NDArray[np.intp] = field(default_factory=_EMPTY)
    x_last: NDArray[np.intp] = field(default_factory=_EMPTY)
    x_face_hi: NDArray[np.intp] = field(default_factory=_EMPTY)
    x_face_lo_inner: NDArray[np.intp] = field(default_factory=_EMPTY)
    x_first_inner: NDArray[np.intp] = field(default_factory=_EMPTY)
    x_last_inner: NDArray[np.intp] = field(default_factory=_EMPTY)
    x_face_hi_inner: NDArray[np.intp] = field(default_factory=_EMPTY)

    y_face_lo: NDArray[np.intp] = field(default_factory=_EMPTY)
    y_first: NDArray[np.intp] = field(default_factory=_EMPTY)
    y_last: NDArray[np.intp] = field(default_factory=_EMPTY)
    y_face_hi: NDArray[np.intp] = field(default_factory=_EMPTY)
    y_face_lo_inner: NDArray[np.intp] = field(default_factory=_EMPTY)
    y_first_inner: NDArray[np.intp] = field(default_factory=_EMPTY)
    y_last_inner: NDArray[np.intp] = field(default_factory=_EMPTY)
    y_face_hi_inner: NDArray[np.intp] = field(default_factory=_EMPTY)

    z_face_lo: NDArray[np.intp] = field(default_factory=_EMPTY)
    z_first: NDArray[np.intp] = field(default_factory=_EMPTY)
    z_last: NDArray[np.intp] = field(default_factory=_EMPTY)
    z_face_hi: NDArray[np.intp] = field(default_factory=_EMPTY)
    z_face_lo_inner: NDArray[np.intp] = field(default_factory=_EMPTY)
    z_first_inner: NDArray[np.intp] = field(default_factory=_EMPTY)
    z_last_inner: NDArray[np.intp] = field(default_factory=_EMPTY)
    z_face_hi_inner: NDArray[np.intp] = field(default_factory=_EMPTY)

    x_normal_bc_mask: NDArray[np.intp] = field(default_factory=_EMPTY)
    y_normal_bc_mask: NDArray[np.intp] = field(default_factory=_EMPTY)
    z_normal_bc_mask: NDArray[np.intp] = field(default_factory=_EMPTY)

    hole_x_bc_mask: NDArray[np.intp] = field(default_factory=_EMPTY)
    hole_y_bc_mask: NDArray[np.intp] = field(default_factory=_EMPTY)
    hole_z_bc_mask: NDArray[np.intp] = field(default_factory=_EMPTY)
    hole_x_bc_interior: NDArray[np.intp] = field(default_factory=_EMPTY)
    hole_y_bc_interior: NDArray[np.intp] = field(default_factory=_EMPTY)
    hole_z_bc_interior: NDArray[np.intp] = field(default_factory=_EMPTY)

    def define_hole_polygon(self, vertices, z_range, params: SimulationParameters) -> None:
        """Append the hole-boundary link masks of one polygon hole
        (src/tdgl3d/mesh/indices.py:136-232).

        Links are appended per call, so several holes accumulate; the interior
        lists keep only links whose own node is an interior node, in link
        order."""
        hole = identify_hole_nodes(vertices, z_range, params.hx, params.hy,
                                   params.Nx, params.Ny, params.Nz)
        full_to_int = np.full(params.dim_x, -1, dtype=np.intp)
        full_to_int[self.interior_to_full] = np.arange(params.n_interior, dtype=np.intp)
        for axis in ("x", "y", "z"):
            links = identify_boundary_links(hole, axis, is_3d=params.is_3d)
            name = f"hole_{axis}_bc_mask"
            setattr(self, name, np.concatenate([getattr(self, name), links]))
            inner = full_to_int[links]
            inner = inner[inner >= 0].astype(np.intp)
            if inner.size:
                iname = f"hole_{axis}_bc_interior"
                setattr(self, iname, np.concatenate([getattr(self, iname), inner]))


def _lin(i, j, k, mj, mk):
    return (np.asarray(i, dtype=np.intp) + mj * np.asarray(j, dtype=np.intp)
            + mk * np.asarray(k, dtype=np.intp))


def construct_indices(params: SimulationParameters) -> GridIndices:
    """Build every index array of :class:`GridIndices`
    (src/tdgl3d/mesh/indices.py:239-450).

    Ordering rules, which callers depend on:

    * ``interior_to_full`` enumerates interior nodes with **k fastest** and
      i slowest (an ``ij``-indexed meshgrid flattened in C order).
    * Each face array enumerates its two free axes with the lower-numbered
      free axis slowest (x faces: j slow, k fast; y faces: i slow, k fast;
      z faces: i slow, j fast); the *inner* variants drop edge nodes.
    * ``*_normal_bc_mask`` is the face at index 0 followed by the face at
      index N-1 (not N) of that axis, over all nodes of the free axes.
    """
    Nx, Ny, Nz = params.Nx, params.Ny, params.Nz
    mj, mk = Nx + 1, (Nx + 1) * (Ny + 1)
    is_3d = Nz > 1
    all_i, all_j = np.arange(Nx + 1), np.arange(Ny + 1)
    all_k = np.arange(Nz + 1) if is_3d else np.zeros(1, dtype=np.intp)
    int_i, int_j = np.arange(1, Nx), np.arange(1, Ny)
    int_k = np.arange(1, Nz) if is_3d else np.zeros(1, dtype=np.intp)

    I, J, K = np.meshgrid(int_i, int_j, int_k, indexing="ij")
    interior_to_full = _lin(I.ravel(), J.ravel(), K.ravel(), mj, mk)

    # bfield_interior: interior-numbering offsets (i-1) + (Nx-1)(j-1) + (Nx-1)(Ny-1)(k-1)
    # of the nodes one layer further in, enumerated with k fastest.
    bi, bj = np.arange(Nx - 2), np.arange(Ny - 2)
    if is_3d:
        BI, BJ, BK = np.meshgrid(bi, bj, np.arange(Nz - 2), indexing="ij")
        bfield_interior = (BI.ravel() + (Nx - 1) * BJ.ravel()
                           + (Nx - 1) * (Ny - 1) * BK.ravel()).astype(np.intp)
    else:
        BI, BJ = np.meshgrid(bi, bj, indexing="ij")
        bfield_interior = (BI.ravel() + (Nx - 1) * BJ.ravel()).astype(np.intp)

    def face(axis: str, value: int, r1, r2):
        A, B = np.meshgrid(r1, r2, indexing="ij")
        a, b = A.ravel(), B.ravel()
        v = np.full(a.size, value, dtype=np.intp)
        if axis == "x":
            return _lin(v, a, b, mj, mk)
        if axis == "y":
            return _lin(a, v, b, mj, mk)
        return _lin(a, b, v, mj, mk)

    out: dict[str, NDArray] = {}
    spec = {
        "x": (Nx, all_j, all_k, int_j, int_k),
        "y": (Ny, all_i, all_k, int_i, int_k),
        "z": (Nz, all_i, all_j, int_i, int_j),
    }
    for axis, (N, a_all, b_all, a_int, b_int) in spec.items():
        if axis == "z" and not is_3d:
            for nm in ("face_lo", "first", "last", "face_hi", "face_lo_inner",
                       "first_inner", "last_inner", "face_hi_inner", "normal_bc_mask"):
                out[f"z_{nm}"] = _EMPTY()
            continue
        pos = {"face_lo": 0, "first": 1, "last": N - 1, "face_hi": N}
        for nm, val in pos.items():
            out[f"{axis}_{nm}"] = face(axis, val, a_all, b_all)
            out[f"{axis}_{nm}_inner"] = face(axis, val, a_int, b_int)
        out[f"{axis}_normal_bc_mask"] = np.concatenate(
            [face(axis, 0, a_all, b_all), face(axis, N - 1, a_all, b_all)])

    return GridIndices(interior_to_full=interior_to_full,
                       bfield_interior=bfield_interior, **out)


# ---------------------------------------------------------------------------
# Holes
# ---------------------------------------------------------------------------

def _crossing_parity(x: NDArray, y: NDArray, vertices) -> NDArray[np.bool_]:
    """Even-odd ray-crossing test, vectorised over many points.

    The per-edge predicate is the one of src/tdgl3d/mesh/holes.py:84-98
    (``y > min(p1y,p2y)``, ``y <= max(p1y,p2y)``, ``x <= max(p1x,p2x)``, then
    ``p1x == p2x`` or ``x <= xinters``), with ``xinters`` evaluated in the same
    floating-point operation order, so points on edges classify identically.
    Horizontal edges never pass the first two tests, so their ``xinters`` is
    never needed.
    """
    verts = [(float(a), float(b)) for a, b in vertices]
    n = len(verts)
    inside = np.zeros(np.broadcast(x, y).shape, dtype=bool)
    for e in range(n):
        p1x, p1y = verts[e]
        p2x, p2y = verts[(e + 1) % n]
        hit = (y > min(p1y, p2y)) & (y <= max(p1y, p2y)) & (x <= max(p1x, p2x))
        if p1x == p2x:
            inside ^= hit
        elif p1y != p2y:
            with np.errstate(invalid="ignore", divide="ignore"):
                xinters = (y - p1y) * (p2x - p1x) / (p2y - p1y) + p1x
            inside ^= hit & (x <= xinters)
    return inside


def point_in_polygon(point, vertices) -> bool:
    """Ray-casting point-in-polygon test (src/tdgl3d/mesh/holes.py:43-100)."""
    x, y = point
    return bool(_crossing_parity(np.float64(x), np.float64(y), vertices))


def identify_hole_nodes(vertices, z_range, grid_spacing_x, grid_spacing_y,
                        Nx, Ny, Nz) -> NDArray[np.bool_]:
    """Boolean mask of shape (Nx+1, Ny+1, Nz+1) of nodes inside a polygon,
    extruded over planes ``z_min..min(z_max, Nz)`` inclusive
    (src/tdgl3d/mesh/holes.py:103-157).  Node (i, j) sits at (i*hx, j*hy)."""
    i = np.arange(Nx + 1)
    j = np.arange(Ny + 1)
    X = (i * float(grid_spacing_x))[:, None]
    Y = (j * float(grid_spacing_y))[None, :]
    plane = _crossing_parity(X, Y, vertices)
    mask = np.zeros((Nx + 1, Ny + 1, Nz + 1), dtype=bool)
    z_min, z_max = z_range
    ks = range(z_min, min(z_max + 1, Nz + 1))
    for k in ks:
        mask[:, :, k] = plane
    return mask


def identify_circular_hole_nodes(center, radius, z_range, grid_spacing_x,
                                 grid_spacing_y, Nx, Ny, Nz) -> NDArray[np.bool_]:
    """Mask of nodes strictly inside a circle (src/tdgl3d/mesh/holes.py:260-311)."""
    cx, cy = center
    X = (np.arange(Nx + 1) * float(grid_spacing_x))[:, None]
    Y = (np.arange(Ny + 1) * float(grid_spacing_y))[None, :]
    plane = np.sqrt((X - cx) ** 2 + (Y - cy) ** 2) < radius
    mask = np.zeros((Nx + 1, Ny + 1, Nz + 1), dtype=bool)
    z_min, z_max = z_range
    for k in range(z_min, min(z_max + 1, Nz + 1)):
        mask[:, :, k] = plane
    return mask


def identify_boundary_links(hole_mask: NDArray[np.bool_], direction: str,
                            is_3d: bool = True) -> NDArray[np.int64]:
    """Full-grid indices of the links whose two end nodes disagree on being
    inside the hole (src/tdgl3d/mesh/holes.py:160-257).

    The link from node n to n + e_d is indexed by n.  Order: x links with i
    fastest then j then k; y links with j fastest then i then k; z links with
    k fastest then j then i.  In 2-D the index drops k, so each link of the
    two planes k=0 and k=1 is listed once per plane.
    """
    Nx, Ny, Nz = (s - 1 for s in hole_mask.shape)
    h = hole_mask
    if direction == "x":
        d = h[:-1, :, :] != h[1:, :, :]            # (i, j, k), i < Nx
        order = d.transpose(2, 1, 0)               # k, j, i  (i fastest)
        kk, jj, ii = np.nonzero(order)
    elif direction == "y":
        d = h[:, :-1, :] != h[:, 1:, :]            # (i, j, k), j < Ny
        order = d.transpose(2, 0, 1)               # k, i, j  (j fastest)
        kk, ii, jj = np.nonzero(order)
    elif direction == "z":
        d = h[:, :, :-1] != h[:, :, 1:]            # (i, j, k), k < Nz
        ii, jj, kk = np.nonzero(d)                 # i, j, k  (k fastest)
    else:
        raise ValueError(f"Invalid direction '{direction}'. Use 'x', 'y', or 'z'.")
    mj, mk = Nx + 1, (Nx + 1) * (Ny + 1)
    if is_3d:
        m = kk * mk + jj * mj + ii
    else:
        m = jj * mj + ii
    return np.asarray(m, dtype=np.int64)


# ---------------------------------------------------------------------------
# Materials
# ---------------------------------------------------------------------------

@dataclass
class MaterialMap:
    """Per-node κ and superconducting mask on the full grid, plus the mask at
    interior nodes (src/tdgl3d/core/material.py:26-112)."""

    kappa: NDArray[np.float64]
    sc_mask: NDArray[np.float64]
    interior_sc_mask: NDArray[np.float64]

    def carve_hole_polygon(self, vertices, z_range, params: SimulationParameters, idx) -> None:
        """Set sc_mask = 0 on the nodes inside a polygon hole
        (src/tdgl3d/core/material.py:43-112).  In 2-D the plane index is
        dropped, so nodes of either plane map onto the single layer."""
        hole = identify_hole_nodes(vertices, z_range, params.hx, params.hy,
                                   params.Nx, params.Ny, params.Nz)
        ii, jj, kk = np.nonzero(hole)
        m = ii + params.mj * jj + (params.mk * kk if params.is_3d else 0)
        self.sc_mask[m] = 0.0
        self.interior_sc_mask = self.sc_mask[idx.interior_to_full]


@dataclass
class Layer:
    """One layer of a stack: thickness in z cells, κ, superconducting or not
    (src/tdgl3d/core/material.py:120-136)."""

    thickness_z: int
    kappa: float
    is_superconductor: bool = True


@dataclass
class Trilayer:
    """Superconductor / insulator / superconductor stack along z
    (src/tdgl3d/core/material.py:139-175)."""

    bottom: Layer
    insulator: Layer
    top: Layer

    def __post_init__(self) -> None:
        if self.insulator.is_superconductor:
            raise ValueError("The insulator layer must have is_superconductor=False.")

    @property
    def Nz(self) -> int:
        return self.bottom.thickness_z + self.insulator.thickness_z + self.top.thickness_z

    def z_ranges(self) -> dict[str, tuple[int, int]]:
        b, i = self.bottom.thickness_z, self.insulator.thickness_z
        return {"bottom": (0, b), "insulator": (b, b + i),
                "top": (b + i, b + i + self.top.thickness_z)}


def build_material_map(params: SimulationParameters, trilayer: Trilayer, idx) -> MaterialMap:
    """Per-plane κ and sc mask of a trilayer (src/tdgl3d/core/material.py:182-254).

    Plane k takes the first layer whose half-open cell range contains k; the
    last plane k = Nz (and any plane no range covers) belongs to the top."""
    if params.Nz != trilayer.Nz:
        raise ValueError(f"params.Nz={params.Nz} does not match trilayer.Nz={trilayer.Nz}")
    layers = {"bottom": trilayer.bottom, "insulator": trilayer.insulator, "top": trilayer.top}
    plane_kappa = np.empty(params.Nz + 1)
    plane_sc = np.empty(params.Nz + 1)
    ranges = list(trilayer.z_ranges().items())
    for k in range(params.Nz + 1):
        name = next((nm for nm, (a, b) in ranges if a <= k < b), "top")
        plane_kappa[k] = layers[name].kappa
        plane_sc[k] = 1.0 if layers[name].is_superconductor else 0.0
    mk = params.mk
    kappa_full = np.repeat(plane_kappa, mk)[: params.dim_x].astype(np.float64)
    sc_full = np.repeat(plane_sc, mk)[: params.dim_x].astype(np.float64)
    return MaterialMap(kappa=kappa_full, sc_mask=sc_full,
                       interior_sc_mask=sc_full[idx.interior_to_full])


def polygon_vertices(vertices: Sequence) -> list[tuple[float, float]]:
    return [(float(a), float(b)) for a, b in vertices]
