"""Generate golden fixtures for the analysis functions from the tdgl3d
reference (src/tdgl3d/analysis/vortex_counting.py, convergence.py).

Run where the reference source tree is available (imported read-only from
``<reference>/src``)::

    python tests/golden/make_analysis_golden.py --reference <path to the tdgl3d checkout>

Writes ``analysis.npz`` next to this script: seeded states with phase
windings (2-D and a 3-D film with a hole), the reference's plaquette vortex
counts, hole flux, core positions and polygon fluxoid per slice, and the
convergence metrics / steady-state answers on synthetic trajectories.
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def vortex_state(params, centers, sc=None, rng=None, phi_scale=0.0):
    """psi = prod_v tanh(r_v / 2) exp(i s_v theta_v) per interior node (reference
    interior order: k fastest), centers (x0, y0, sign, dx_per_k) in interior
    index units; phi = phi_scale * N(0, 1)."""
    nx, ny = params.Nx - 1, params.Ny - 1
    nz = max(params.Nz - 1, 1)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    psi = np.ones((nx, ny, nz), dtype=np.complex128)
    for x0, y0, sgn, drift in centers:
        dx = i - (x0 + drift * k)
        dy = j - y0
        r = np.sqrt(dx ** 2 + dy ** 2)
        psi *= np.tanh(r / 2.0) * np.exp(1j * sgn * np.arctan2(dy, dx))
    psi = psi.reshape(-1)
    if sc is not None:
        psi = psi * sc
    n = params.n_interior
    x = np.zeros(params.n_state, dtype=np.complex128)
    x[:n] = psi
    if phi_scale:
        x[n:] = phi_scale * rng.standard_normal(params.n_state - n)
    return x


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("TDGL3D_REFERENCE"),
                    help="checkout of omedeiro/nanowire_tdgl (its src/ is imported); or set TDGL3D_REFERENCE")
    a = ap.parse_args()
    if not a.reference:
        ap.error("--reference (or TDGL3D_REFERENCE) is required")
    sys.path.insert(0, os.path.join(a.reference, "src"))
    import tdgl3d
    from tdgl3d.analysis.convergence import check_steady_state, compute_convergence_metrics
    from tdgl3d.analysis.vortex_counting import (count_hole_flux_quanta, count_vortices_plaquette,
                                                 count_vortices_polygon, find_vortex_cores)
    from tdgl3d.core.solution import Solution

    out = {}
    rng = np.random.default_rng(21)

    # --- 2-D: two vortices of opposite sign -----------------------------------
    p2 = tdgl3d.SimulationParameters(Nx=30, Ny=30, hx=1.0, hy=1.0, hz=1.0, kappa=2.0)
    d2 = tdgl3d.Device(p2, applied_field=tdgl3d.AppliedField(Bz=0.0))
    x2 = vortex_state(p2, [(9.3, 14.2, 1, 0.0), (19.6, 13.7, -1, 0.0)])
    s2 = Solution(times=np.array([0.0]), states=x2[:, None], params=p2, idx=d2.idx, device=d2)
    out["v2_x"] = x2
    for tag, (wt, mt) in {"a": (0.8, 0.02), "b": (0.5, 0.02), "c": (0.8, 0.3)}.items():
        n, pos, w = count_vortices_plaquette(s2, d2, slice_z=0, step=0, winding_threshold=wt, mask_threshold=mt)
        out[f"v2_{tag}_n"] = np.array(n)
        out[f"v2_{tag}_pos"] = np.asarray(pos, dtype=float).reshape(-1, 2)
        out[f"v2_{tag}_w"] = np.asarray(w, dtype=float)

    # --- 3-D film with a hole, vortices drifting with z ----------------------
    p3 = tdgl3d.SimulationParameters(Nx=24, Ny=20, Nz=5, hx=0.5, hy=0.5, hz=0.5, kappa=2.0)
    d3 = tdgl3d.Device(p3, applied_field=tdgl3d.AppliedField(Bz=0.4, t_on_fraction=1.0))
    d3.add_hole([(7.0, 3.0), (9.0, 3.0), (9.0, 5.5), (7.0, 5.5)])
    sc3 = d3.material.interior_sc_mask
    x3 = vortex_state(p3, [(5.2, 8.4, 1, 0.7), (11.5, 13.1, -1, -0.4), (8.1, 14.6, 1, 0.0)], sc=sc3, rng=rng,
                      phi_scale=0.05)
    s3 = Solution(times=np.array([0.0, 1.0]), states=np.stack([x3 * 0.5, x3], axis=1), params=p3, idx=d3.idx,
                  device=d3)
    out["v3_x"] = x3
    ns = p3.Nz - 1
    for k in range(ns):
        n, pos, w = count_vortices_plaquette(s3, d3, slice_z=k, step=-1)
        out[f"v3_{k}_n"] = np.array(n)
        out[f"v3_{k}_pos"] = np.asarray(pos, dtype=float).reshape(-1, 2)
        out[f"v3_{k}_w"] = np.asarray(w, dtype=float)
        out[f"v3_{k}_flux"] = np.array(count_hole_flux_quanta(s3, d3, (13.0, 17.0, 5.0, 9.0), slice_z=k, step=-1))
        out[f"v3_{k}_cores"] = np.asarray(find_vortex_cores(s3, d3, slice_z=k, step=-1, threshold=0.1,
                                                             separation=2), dtype=float).reshape(-1, 2)
        out[f"v3_{k}_poly"] = np.array(count_vortices_polygon(s3, d3, np.array([[2, 2], [16, 2], [16, 18], [2, 18]]),
                                                              slice_z=k, step=-1))

    # --- convergence: relaxing trajectory on the holed film ------------------
    nt = 40
    times = np.linspace(0.0, 19.5, nt)
    n3 = p3.n_interior
    base = x3.copy()
    states = np.zeros((p3.n_state, nt), dtype=np.complex128)
    for t_i, t in enumerate(times):
        amp = 1.0 - 0.5 * np.exp(-t / 2.0)
        st = base.copy()
        st[:n3] = base[:n3] * amp
        st[n3:] = base[n3:] * (1.0 + 0.3 * np.exp(-t / 3.0))
        states[:, t_i] = st
    sc_sol = Solution(times=times, states=states, params=p3, idx=d3.idx, device=d3)
    out["conv_times"] = times
    out["conv_states"] = states
    for tag, (dev, step, win) in {"a": (d3, -1, 10), "b": (d3, 25, 5), "c": (None, -1, 10), "d": (d3, 3, 10)}.items():
        m = compute_convergence_metrics(sc_sol, dev, step=step, window_size=win)
        for key in ("psi2_mean_current", "psi2_mean_past", "psi2_rel_change", "current_mean_current",
                    "current_mean_past", "current_rel_change"):
            if key in m:
                out[f"conv_{tag}_{key}"] = np.array(m[key])
    for tag, kw in {"a": dict(window_size=5, psi_threshold=1e-3, current_threshold=1e-3, start_step=10),
                    "b": dict(window_size=10, psi_threshold=1e-4, current_threshold=1e-4, start_step=20),
                    "c": dict(window_size=5, psi_threshold=1e-2, current_threshold=1e-2, start_step=5)}.items():
        dev = None if tag == "c" else d3
        is_steady, steady_step, m = check_steady_state(sc_sol, dev, **kw)
        out[f"steady_{tag}_is"] = np.array(bool(is_steady))
        out[f"steady_{tag}_step"] = np.array(steady_step)
        out[f"steady_{tag}_time"] = np.array(m.get("steady_time", np.nan))
        out[f"steady_{tag}_psi2_rel_change"] = np.array(m["psi2_rel_change"])

    path = os.path.join(HERE, "analysis.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
