"""nanowire_tdgl_b200 — B200-native trapezoidal stepper for the tdgl3d TDGL model.

Public names mirror the tdgl3d package (src/tdgl3d/__init__.py:9-46) for the
time-stepping path: set up a :class:`Device`, then call :func:`solve` (or the
lower-level ``trapezoidal`` / ``newton_gcr_trap`` / ``tgcr_matrix_free_trap``
/ ``eval_f``).  The numerics run in sm_100a CUDA kernels behind the C ABI of
``include/tdgl_b200.h``; the Python layer only stages data.
"""

from .geometry import (GridIndices, Layer, MaterialMap, SimulationParameters, Trilayer,
                       build_material_map, construct_indices, identify_boundary_links,
                       identify_circular_hole_nodes, identify_hole_nodes, point_in_polygon)
from .model import (AppliedField, BoundaryVectors, Device, StateVector,
                    build_boundary_field_vectors)

__version__ = "0.1.0"

__all__ = [
    "SimulationParameters", "GridIndices", "construct_indices", "MaterialMap", "Layer",
    "Trilayer", "build_material_map", "point_in_polygon", "identify_hole_nodes",
    "identify_boundary_links", "identify_circular_hole_nodes", "AppliedField",
    "BoundaryVectors", "build_boundary_field_vectors", "Device", "StateVector",
]
from .solvers import (DeviceRHS, FieldSchedule, eval_f, forward_euler, make_eval_f, newton_gcr_trap, solve,
                      tgcr_matrix_free_trap, trapezoidal)
from .solution import Solution
from .hdf5 import load_solution, save_solution

__all__ += ["DeviceRHS", "FieldSchedule", "eval_f", "forward_euler", "make_eval_f", "newton_gcr_trap",
            "solve", "tgcr_matrix_free_trap", "trapezoidal", "Solution"]
from .adjoint import box_mean_psi2, rhs, trapezoidal_gradient

__all__ += ["box_mean_psi2", "rhs", "trapezoidal_gradient"]
from .batch import BatchedTrapezoidal

__all__ += ["BatchedTrapezoidal", "load_solution", "save_solution"]
from .analysis import (check_steady_state, compute_convergence_metrics, count_hole_flux_quanta,
                       count_vortices_plaquette, count_vortices_polygon, find_vortex_cores, plaquette_windings)

__all__ += ["check_steady_state", "compute_convergence_metrics", "count_hole_flux_quanta",
            "count_vortices_plaquette", "count_vortices_polygon", "find_vortex_cores", "plaquette_windings"]
