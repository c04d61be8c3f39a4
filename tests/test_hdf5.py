"""HDF5 result files (``Solution.save`` / ``Solution.load`` and
``save_solution`` / ``load_solution``) in the reference's two layouts.

h5py is not installed in this image, so the round trips run against a small
in-memory stand-in for the part of h5py's API that the layouts use (File,
Group, Dataset, attrs); without it the calls raise ModuleNotFoundError, as
the reference's do.  The reference's own check of this path
(tests/test_hole_bc_smoke.py:163-199) saves a holed device's solution and
compares the loaded hole masks.
"""

import importlib.util
import sys
import types

import numpy as np
import pytest


class _Dataset:
    def __init__(self, data):
        self._a = np.array(data, copy=True)

    def __getitem__(self, key):
        return np.array(self._a[key], copy=True)


class _Group:
    def __init__(self):
        self.attrs = {}
        self._items = {}

    def create_dataset(self, name, data):
        assert name not in self._items
        self._items[name] = _Dataset(data)
        return self._items[name]

    def create_group(self, name):
        assert name not in self._items
        self._items[name] = _Group()
        return self._items[name]

    def __getitem__(self, name):
        return self._items[name]

    def __contains__(self, name):
        return name in self._items

    def keys(self):
        return list(self._items)


class _File:
    store: dict = {}

    def __init__(self, name, mode="r"):
        key = str(name)
        if mode == "w":
            _File.store[key] = _Group()
        elif mode != "r" or key not in _File.store:
            raise OSError(f"cannot open {key} with mode {mode}")
        self.root = _File.store[key]

    def __enter__(self):
        return self.root

    def __exit__(self, *exc):
        return False


@pytest.fixture
def fake_h5py(monkeypatch):
    mod = types.ModuleType("h5py")
    mod.File, mod.Group, mod.Dataset = _File, _Group, _Dataset
    _File.store = {}
    monkeypatch.setitem(sys.modules, "h5py", mod)
    return mod


def _solution(periodic=False, hole=True):
    import nanowire_tdgl_b200 as tb
    p = tb.SimulationParameters(Nx=8, Ny=8, Nz=4, hx=1.0, hy=1.0, hz=1.0, kappa=2.0,
                                periodic_x=periodic, periodic_y=periodic)
    dev = tb.Device(p)
    if hole:
        dev.add_hole([(3.0, 3.0), (5.0, 3.0), (5.0, 5.0), (3.0, 5.0)])
    rng = np.random.default_rng(4)
    states = rng.standard_normal((p.n_state, 3)) + 1j * rng.standard_normal((p.n_state, 3))
    meta = {"method": "trapezoidal", "dt": 0.1, "n_saved": 3, "kappa_map": np.linspace(0.0, 1.0, 5),
            "solver": {"name": "gmres", "tol": 1e-6, "history": np.arange(4.0)}}
    return tb.Solution(times=np.array([0.0, 0.1, 0.2]), states=states, params=p, idx=dev.idx, device=dev,
                       metadata=meta)


def _idx_arrays(idx):
    return {k: getattr(idx, k) for k in dir(idx)
            if not k.startswith("_") and isinstance(getattr(idx, k), np.ndarray)}


def test_solution_save_load_keeps_indices_and_metadata(fake_h5py, tmp_path):
    import nanowire_tdgl_b200 as tb
    sol = _solution()
    assert len(sol.idx.hole_x_bc_mask) > 0 and len(sol.idx.hole_y_bc_mask) > 0
    path = tmp_path / "run.h5"
    sol.save(path)
    back = tb.Solution.load(path)
    assert back.device is None
    assert np.array_equal(back.times, sol.times) and np.array_equal(back.states, sol.states)
    for k in ("Nx", "Ny", "Nz", "hx", "hy", "hz", "kappa"):
        assert getattr(back.params, k) == getattr(sol.params, k)
    want = _idx_arrays(sol.idx)
    got = _idx_arrays(back.idx)
    assert set(want) <= set(got)
    for k, v in want.items():
        assert np.array_equal(got[k], v), k
    m = back.metadata
    assert m["method"] == "trapezoidal" and m["dt"] == 0.1 and m["n_saved"] == 3
    assert np.array_equal(m["kappa_map"], sol.metadata["kappa_map"])
    assert m["solver"]["name"] == "gmres" and m["solver"]["tol"] == 1e-6
    assert np.array_equal(m["solver"]["history"], np.arange(4.0))
    # the file's layout is the reference's
    root = _File.store[str(path)]
    assert set(root.keys()) == {"times", "states", "params", "idx", "metadata"}
    assert set(root["params"].attrs) == {"Nx", "Ny", "Nz", "hx", "hy", "hz", "kappa"}


def test_solution_without_metadata(fake_h5py, tmp_path):
    import nanowire_tdgl_b200 as tb
    sol = _solution(hole=False)
    sol.metadata = None
    sol.save(tmp_path / "a.h5")
    back = tb.Solution.load(tmp_path / "a.h5")
    assert back.metadata is None and np.array_equal(back.states, sol.states)


def test_save_solution_layout_rebuilds_indices(fake_h5py, tmp_path):
    import nanowire_tdgl_b200 as tb
    sol = _solution(periodic=True, hole=False)
    out = tb.save_solution(sol, str(tmp_path / "b.h5"))
    assert out == tmp_path / "b.h5"
    root = _File.store[str(out)]
    assert set(root.keys()) == {"times", "states_real", "states_imag", "params"}
    back = tb.load_solution(out)
    assert np.array_equal(back.states, sol.states) and np.array_equal(back.times, sol.times)
    assert back.params.periodic_x and back.params.periodic_y and not back.params.periodic_z
    ref = tb.construct_indices(back.params)
    for k, v in _idx_arrays(ref).items():
        assert np.array_equal(getattr(back.idx, k), v), k


@pytest.mark.skipif(importlib.util.find_spec("h5py") is not None, reason="h5py is installed")
def test_without_h5py_the_calls_raise(monkeypatch, tmp_path):
    import nanowire_tdgl_b200 as tb
    monkeypatch.delitem(sys.modules, "h5py", raising=False)
    sol = _solution(hole=False)
    with pytest.raises(ModuleNotFoundError):
        sol.save(tmp_path / "c.h5")
    with pytest.raises(ModuleNotFoundError):
        tb.Solution.load(tmp_path / "c.h5")
    with pytest.raises(ModuleNotFoundError):
        tb.save_solution(sol, tmp_path / "c.h5")
    with pytest.raises(ModuleNotFoundError):
        tb.load_solution(tmp_path / "c.h5")
