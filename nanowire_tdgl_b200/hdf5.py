"""HDF5 result files in the two layouts tdgl3d writes.

* ``Solution.save`` / ``Solution.load`` (src/tdgl3d/core/solution.py:400-549):
  ``times``, complex ``states``, group ``params`` (attributes Nx, Ny, Nz, hx,
  hy, hz, kappa), group ``idx`` (every public array of ``GridIndices`` as a
  dataset, scalars as attributes, so hole masks survive), optional group
  ``metadata`` (scalars as attributes, arrays as datasets, one level of
  nested dicts as subgroups).
* ``save_solution`` / ``load_solution`` (src/tdgl3d/io/hdf5.py:14-79):
  ``times``, ``states_real`` and ``states_imag``, group ``params`` with the
  periodic flags as well; loading rebuilds the indices from the parameters
  (``construct_indices``; holes are not stored in this layout).

The layouts are the reference's so that files move between the two
packages either way.  h5py is imported when a file is read or written, as
the reference does; without it both raise ``ModuleNotFoundError``.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np

_PARAM_KEYS = ("Nx", "Ny", "Nz", "hx", "hy", "hz", "kappa")
_PERIODIC_KEYS = ("periodic_x", "periodic_y", "periodic_z")
_SCALARS = (str, int, float, bool, np.integer, np.floating, np.bool_)


def _params_from_attrs(attrs, periodic: bool):
    from .geometry import SimulationParameters
    kw = {k: (int(attrs[k]) if k in ("Nx", "Ny", "Nz") else float(attrs[k])) for k in _PARAM_KEYS}
    if periodic:
        kw.update({k: bool(attrs[k]) for k in _PERIODIC_KEYS})
    return SimulationParameters(**kw)


def _write_dict(h5py, grp, items: dict, depth: int) -> None:
    for key, val in items.items():
        if isinstance(val, _SCALARS):
            grp.attrs[key] = val
        elif isinstance(val, np.ndarray):
            grp.create_dataset(key, data=val)
        elif isinstance(val, dict) and depth > 0:
            _write_dict(h5py, grp.create_group(key), val, depth - 1)


def _read_dict(h5py, grp, depth: int) -> dict:
    out = {k: grp.attrs[k] for k in grp.attrs}
    for key in grp.keys():
        item = grp[key]
        if isinstance(item, h5py.Dataset):
            out[key] = item[:]
        elif isinstance(item, h5py.Group) and depth > 0:
            out[key] = _read_dict(h5py, item, depth - 1)
    return out


def save_full(solution, filename) -> None:
    """``Solution.save``: the solution.py layout (indices and metadata
    included)."""
    import h5py
    with h5py.File(filename, "w") as f:
        f.create_dataset("times", data=np.asarray(solution.times))
        f.create_dataset("states", data=np.asarray(solution.states))
        grp = f.create_group("params")
        for key in _PARAM_KEYS:
            grp.attrs[key] = getattr(solution.params, key)
        gidx = f.create_group("idx")
        for key in dir(solution.idx):
            if key.startswith("_"):
                continue
            val = getattr(solution.idx, key)
            if isinstance(val, np.ndarray):
                gidx.create_dataset(key, data=val)
            elif isinstance(val, (int, float, bool)):
                gidx.attrs[key] = val
        if solution.metadata is not None:
            _write_dict(h5py, f.create_group("metadata"), solution.metadata, 1)


def load_full(filename):
    """``Solution.load``: the solution.py layout; the device is not stored
    (``device`` is None)."""
    import h5py
    from .geometry import GridIndices
    from .solution import Solution
    with h5py.File(filename, "r") as f:
        times = f["times"][:]
        states = f["states"][:]
        params = _params_from_attrs(f["params"].attrs, periodic=False)
        gidx = f["idx"]
        idx = GridIndices(**{key: gidx[key][:] for key in gidx.keys()})
        metadata = _read_dict(h5py, f["metadata"], 1) if "metadata" in f else None
    return Solution(times=times, states=states, params=params, idx=idx, device=None, metadata=metadata)


def save_solution(solution, filepath) -> Path:
    """src/tdgl3d/io/hdf5.py:14-42: times, real and imaginary states, all
    parameters; returns the path written."""
    import h5py
    filepath = Path(filepath)
    states = np.asarray(solution.states)
    with h5py.File(filepath, "w") as f:
        f.create_dataset("times", data=np.asarray(solution.times))
        f.create_dataset("states_real", data=np.real(states))
        f.create_dataset("states_imag", data=np.imag(states))
        grp = f.create_group("params")
        for key in _PARAM_KEYS + _PERIODIC_KEYS:
            grp.attrs[key] = getattr(solution.params, key)
    return filepath


def load_solution(filepath):
    """src/tdgl3d/io/hdf5.py:45-79: the states and parameters of a
    ``save_solution`` file, with the indices rebuilt from the parameters."""
    import h5py
    from .geometry import construct_indices
    from .solution import Solution
    with h5py.File(Path(filepath), "r") as f:
        times = f["times"][:]
        states = f["states_real"][:] + 1j * f["states_imag"][:]
        params = _params_from_attrs(f["params"].attrs, periodic=True)
    return Solution(times=times, states=states, params=params, idx=construct_indices(params))
