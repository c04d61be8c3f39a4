"""Analysis functions (vortex counting, steady-state check) against golden
answers the reference produced (tests/golden/make_analysis_golden.py): the
CPU oracle and the host-side functions here, the device kernels with -m gpu."""

import os

import numpy as np
import pytest

from oracle import tdgl_analysis_oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "analysis.npz"))


def _dev2():
    import nanowire_tdgl_b200 as tb
    p = tb.SimulationParameters(Nx=30, Ny=30, hx=1.0, hy=1.0, hz=1.0, kappa=2.0)
    return tb.Device(p, applied_field=tb.AppliedField(Bz=0.0))


def _dev3():
    import nanowire_tdgl_b200 as tb
    p = tb.SimulationParameters(Nx=24, Ny=20, Nz=5, hx=0.5, hy=0.5, hz=0.5, kappa=2.0)
    d = tb.Device(p, applied_field=tb.AppliedField(Bz=0.4, t_on_fraction=1.0))
    d.add_hole([(7.0, 3.0), (9.0, 3.0), (9.0, 5.5), (7.0, 5.5)])
    return d


def _sol(dev, times, states):
    import nanowire_tdgl_b200 as tb
    return tb.Solution(times=np.asarray(times), states=np.asarray(states), params=dev.params, idx=dev.idx,
                       device=dev)


V2 = {"a": (0.8, 0.02), "b": (0.5, 0.02), "c": (0.8, 0.3)}


def _check_count(res, tag):
    n, pos, w = res
    assert n == int(G[f"{tag}_n"])
    assert np.array_equal(np.asarray(pos).reshape(-1, 2), G[f"{tag}_pos"])
    assert np.allclose(w, G[f"{tag}_w"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("tag", list(V2))
def test_oracle_plaquette_2d(tag):
    wt, mt = V2[tag]
    x = G["v2_x"]
    _check_count(orc.count_vortices_plaquette(x[:29 * 29], 30, 30, 1, 0, wt, mt), f"v2_{tag}")


def test_oracle_plaquette_3d_slices():
    d = _dev3()
    p = d.params
    x = G["v3_x"]
    for k in range(p.Nz - 1):
        _check_count(orc.count_vortices_plaquette(x[:p.n_interior], p.Nx, p.Ny, p.Nz, k), f"v3_{k}")


def test_oracle_psi2_means_against_golden():
    d = _dev3()
    n = d.params.n_interior
    S = G["conv_states"]
    sc = d.material.interior_sc_mask
    J0 = (np.zeros(n), np.zeros(n), np.zeros(n))
    for tag, step, win, with_sc in (("a", 39, 10, True), ("b", 25, 5, True), ("c", 39, 10, False)):
        cur = orc.masked_means(S[:n, step], J0, sc if with_sc else None)[0]
        past = orc.masked_means(S[:n, max(0, step - win)], J0, sc if with_sc else None)[0]
        assert abs(cur - float(G[f"conv_{tag}_psi2_mean_current"])) < 1e-13
        assert abs(past - float(G[f"conv_{tag}_psi2_mean_past"])) < 1e-13


def test_host_polygon_and_cores_against_golden():
    import nanowire_tdgl_b200 as tb
    d = _dev3()
    x = G["v3_x"]
    sol = _sol(d, [0.0, 1.0], np.stack([x * 0.5, x], axis=1))
    poly = np.array([[2, 2], [16, 2], [16, 18], [2, 18]])
    for k in range(d.params.Nz - 1):
        assert abs(tb.count_vortices_polygon(sol, d, poly, slice_z=k, step=-1) - float(G[f"v3_{k}_poly"])) < 1e-12
        cores = tb.find_vortex_cores(sol, d, slice_z=k, step=-1, threshold=0.1, separation=2)
        assert np.array_equal(cores.reshape(-1, 2), G[f"v3_{k}_cores"])


def test_solution_methods_dispatch_like_the_reference(monkeypatch):
    """Solution.count_vortices / check_steady_state (solution.py:302-396):
    the host methods give the golden answers, the device ones are forwarded
    with the caller's arguments, bad methods raise ValueError."""
    from nanowire_tdgl_b200 import analysis
    d = _dev3()
    x = G["v3_x"]
    sol = _sol(d, [0.0, 1.0], np.stack([x * 0.5, x], axis=1))
    poly = np.array([[2, 2], [16, 2], [16, 18], [2, 18]])
    got = sol.count_vortices(d, slice_z=1, method="polygon", polygon_points=poly)
    assert abs(got - float(G["v3_1_poly"])) < 1e-12
    cores = sol.count_vortices(d, slice_z=1, method="cores", threshold=0.1, separation=2)
    assert np.array_equal(cores.reshape(-1, 2), G["v3_1_cores"])
    calls = []
    monkeypatch.setattr(analysis, "count_vortices_plaquette", lambda *a, **k: calls.append(("plaq", a, k)) or 7)
    monkeypatch.setattr(analysis, "check_steady_state", lambda *a, **k: calls.append(("steady", a, k)) or 8)
    assert sol.count_vortices(d, 2, 0, winding_threshold=0.5) == 7
    assert sol.check_steady_state(d, 5, 1e-3, 1e-2, 3) == 8
    assert calls == [("plaq", (sol, d, 2, 0), {"winding_threshold": 0.5}),
                     ("steady", (sol, d, 5, 1e-3, 1e-2, 3), {})]
    with pytest.raises(ValueError):
        sol.count_vortices(d, method="polygon")
    with pytest.raises(ValueError):
        sol.count_vortices(d, method="other")


@pytest.mark.gpu
def test_device_plaquette_windings_match_oracle():
    import nanowire_tdgl_b200 as tb
    d = _dev3()
    p = d.params
    x = G["v3_x"]
    sol = _sol(d, [0.0], x[:, None])
    w = tb.plaquette_windings(sol, step=0, mask_threshold=0.02, device=d)
    ref = orc.plaquette_windings(x[:p.n_interior], p.Nx, p.Ny, p.Nz, 0.02)
    assert w.shape == ref.shape
    assert np.array_equal(np.isnan(w), np.isnan(ref))
    assert np.nanmax(np.abs(w - ref)) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("tag", list(V2))
def test_device_count_vortices_2d(tag):
    import nanowire_tdgl_b200 as tb
    d = _dev2()
    sol = _sol(d, [0.0], G["v2_x"][:, None])
    wt, mt = V2[tag]
    _check_count(tb.count_vortices_plaquette(sol, d, slice_z=0, step=0, winding_threshold=wt, mask_threshold=mt),
                 f"v2_{tag}")


@pytest.mark.gpu
def test_device_count_vortices_3d_and_hole_flux():
    import nanowire_tdgl_b200 as tb
    d = _dev3()
    x = G["v3_x"]
    sol = _sol(d, [0.0, 1.0], np.stack([x * 0.5, x], axis=1))
    for k in range(d.params.Nz - 1):
        _check_count(tb.count_vortices_plaquette(sol, d, slice_z=k, step=-1), f"v3_{k}")
        flux = tb.count_hole_flux_quanta(sol, d, (13.0, 17.0, 5.0, 9.0), slice_z=k, step=-1)
        assert abs(flux - float(G[f"v3_{k}_flux"])) < 1e-10


@pytest.mark.gpu
def test_device_convergence_metrics_match_reference():
    import nanowire_tdgl_b200 as tb
    d = _dev3()
    sol = _sol(d, G["conv_times"], G["conv_states"])
    for tag, dev, step, win in (("a", d, -1, 10), ("b", d, 25, 5), ("c", None, -1, 10), ("d", d, 3, 10)):
        m = tb.compute_convergence_metrics(sol, dev, step=step, window_size=win)
        for key in ("psi2_mean_current", "psi2_mean_past", "psi2_rel_change"):
            ref = float(G[f"conv_{tag}_{key}"])
            assert abs(m[key] - ref) <= 1e-12 * max(1.0, abs(ref)), (tag, key)
        assert ("current_error" in m) == (dev is not None)
        assert not any(k.startswith("current_mean") for k in m)


@pytest.mark.gpu
def test_device_check_steady_state_matches_reference():
    import nanowire_tdgl_b200 as tb
    d = _dev3()
    sol = _sol(d, G["conv_times"], G["conv_states"])
    cases = {"a": (d, dict(window_size=5, psi_threshold=1e-3, current_threshold=1e-3, start_step=10)),
             "b": (d, dict(window_size=10, psi_threshold=1e-4, current_threshold=1e-4, start_step=20)),
             "c": (None, dict(window_size=5, psi_threshold=1e-2, current_threshold=1e-2, start_step=5))}
    for tag, (dev, kw) in cases.items():
        ok, step, m = tb.check_steady_state(sol, dev, **kw)
        assert ok == bool(G[f"steady_{tag}_is"]) and step == int(G[f"steady_{tag}_step"])
        if ok:
            assert m["steady_time"] == float(G[f"steady_{tag}_time"]) and m["steady_step"] == step
        assert abs(m["psi2_rel_change"] - float(G[f"steady_{tag}_psi2_rel_change"])) < 1e-12


@pytest.mark.gpu
def test_device_current_means_match_oracle():
    """include_current=True: mean |J_s| over the superconducting nodes, against
    the oracle's supercurrent (pinned to the reference's observables)."""
    import nanowire_tdgl_b200 as tb
    from oracle import tdgl_oracle as o
    d = _dev3()
    S = G["conv_states"]
    sol = _sol(d, G["conv_times"], S)
    m = tb.compute_convergence_metrics(sol, d, step=-1, window_size=10, include_current=True)
    g = o.make_grid(d.params, d.idx, d.material)
    n = d.params.n_interior
    sc = d.material.interior_sc_mask
    for step, key in ((39, "current_mean_current"), (29, "current_mean_past")):
        J = o.supercurrent_density(S[:, step], g)
        ref = orc.masked_means(S[:n, step], J, sc)[1]
        assert abs(m[key] - ref) < 1e-12 * max(1.0, abs(ref))
    assert "current_error" not in m and "current_rel_change" in m


@pytest.mark.gpu
def test_device_plaquettes_on_a_grid_without_plaquettes():
    """Nx = 2: one interior column, no plaquettes; the kernel writes nothing
    and the count is zero, as in the reference's empty scan."""
    import nanowire_tdgl_b200 as tb
    p = tb.SimulationParameters(Nx=2, Ny=5, Nz=3, hx=0.5, hy=0.5, hz=0.5, kappa=2.0)
    d = tb.Device(p)
    x = d.initial_state().data
    sol = _sol(d, [0.0], x[:, None])
    w = tb.plaquette_windings(sol, step=0, device=d)
    assert w.shape == (2, 0, 3)
    n, pos, wind = tb.count_vortices_plaquette(sol, d, slice_z=1, step=0)
    assert n == 0 and pos.shape == (0, 2) and wind.shape == (0,)
    m = tb.compute_convergence_metrics(sol, d, step=0, window_size=1)
    assert m["psi2_mean_current"] == pytest.approx(1.0) and m["psi2_rel_change"] == 0.0
