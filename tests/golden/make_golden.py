"""Generate golden fixtures from the tdgl3d reference implementation.

Run in a container where the reference source tree is mounted (it is imported
read-only from ``<reference>/src``)::

    python tests/golden/make_golden.py --reference <path to the tdgl3d checkout>

It writes small ``.npz`` files next to this script.  The fixtures pin the CPU
oracle (``oracle/tdgl_oracle.py``) and the device path to the reference's own
outputs: integer index maps and hole/material masks, ``eval_f`` on seeded
states over the boundary-condition variants, TGCR / Newton answers, a 101-step
trapezoidal trajectory at the 24x24x8-interior film, short trajectories of the
other geometry variants, a forward-Euler run, and the observables
(|psi|^2, B with boundary conditions, J_s without).

Nothing at test time imports the reference; only these files are read.
"""

from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

IDX_FIELDS = [
    "interior_to_full", "bfield_interior",
    "x_face_lo", "x_first", "x_last", "x_face_hi",
    "x_face_lo_inner", "x_first_inner", "x_last_inner", "x_face_hi_inner",
    "y_face_lo", "y_first", "y_last", "y_face_hi",
    "y_face_lo_inner", "y_first_inner", "y_last_inner", "y_face_hi_inner",
    "z_face_lo", "z_first", "z_last", "z_face_hi",
    "z_face_lo_inner", "z_first_inner", "z_last_inner", "z_face_hi_inner",
    "x_normal_bc_mask", "y_normal_bc_mask", "z_normal_bc_mask",
    "hole_x_bc_mask", "hole_y_bc_mask", "hole_z_bc_mask",
    "hole_x_bc_interior", "hole_y_bc_interior", "hole_z_bc_interior",
]

# name -> geometry/field description shared by the index, RHS and trajectory
# fixtures.  Holes are (vertices, z_range or None).
CASES = {
    "3d_basic": dict(p=dict(Nx=6, Ny=5, Nz=4, hx=0.5, hy=0.6, hz=0.7, kappa=2.0), B=(0.1, 0.2, 0.3)),
    "2d_basic": dict(p=dict(Nx=7, Ny=6, Nz=1, hx=0.5, hy=0.4, kappa=1.5), B=(0.2, 0.3, 0.4)),
    "3d_periodic_x": dict(p=dict(Nx=6, Ny=5, Nz=4, hx=0.5, hy=0.5, hz=0.5, kappa=2.0, periodic_x=True), B=(0.1, 0.2, 0.3)),
    "3d_periodic_yz": dict(p=dict(Nx=5, Ny=6, Nz=5, hx=0.5, hy=0.5, hz=0.5, kappa=2.0, periodic_y=True, periodic_z=True), B=(0.3, -0.2, 0.1)),
    "2d_periodic_xy": dict(p=dict(Nx=6, Ny=6, Nz=1, hx=1.0, hy=1.0, kappa=2.0, periodic_x=True, periodic_y=True), B=(0.0, 0.0, 0.5)),
    "3d_small_nx2": dict(p=dict(Nx=2, Ny=3, Nz=3, hx=0.5, hy=0.5, hz=0.5, kappa=2.0), B=(0.2, 0.1, 0.3)),
    "3d_hole": dict(p=dict(Nx=12, Ny=12, Nz=4, hx=0.5, hy=0.5, hz=0.5, kappa=2.0), B=(0.0, 0.0, 0.5),
                    holes=[([(2.0, 2.0), (4.0, 2.0), (4.0, 4.0), (2.0, 4.0)], None)]),
    "3d_hole_partial_z": dict(p=dict(Nx=12, Ny=10, Nz=5, hx=0.5, hy=0.5, hz=0.5, kappa=2.0), B=(0.1, 0.2, 0.4),
                              holes=[([(2.0, 1.5), (4.0, 1.5), (4.0, 3.5), (2.0, 3.5)], (1, 3))]),
    "3d_hole_edge": dict(p=dict(Nx=10, Ny=10, Nz=3, hx=0.5, hy=0.5, hz=0.5, kappa=2.0), B=(0.2, 0.3, 0.4),
                         holes=[([(-1.0, 2.0), (1.5, 2.0), (1.5, 3.5), (-1.0, 3.5)], None),
                                ([(3.0, 3.0), (4.5, 3.5), (3.5, 4.6)], None)]),
    "2d_hole_triangle": dict(p=dict(Nx=12, Ny=11, Nz=1, hx=0.5, hy=0.5, kappa=2.0), B=(0.0, 0.0, 0.6),
                             holes=[([(1.6, 1.5), (4.2, 1.9), (2.7, 4.3)], None)]),
    "trilayer": dict(p=dict(Nx=8, Ny=7, Nz=5, hx=0.5, hy=0.5, hz=0.5, kappa=2.0), B=(0.1, 0.2, 0.3),
                     trilayer=((2, 2.0, True), (1, 3.0, False), (2, 2.5, True))),
    "trilayer_hole": dict(p=dict(Nx=10, Ny=10, Nz=5, hx=0.5, hy=0.5, hz=0.5, kappa=2.0), B=(0.0, 0.0, 0.4),
                          trilayer=((2, 2.0, True), (1, 2.0, False), (2, 2.0, True)),
                          holes=[([(1.5, 1.5), (3.5, 1.5), (3.5, 3.5), (1.5, 3.5)], None)]),
    "continuous_sc": dict(p=dict(Nx=7, Ny=6, Nz=4, hx=0.5, hy=0.5, hz=0.5, kappa=2.0), B=(0.1, 0.1, 0.2),
                          continuous=True),
    "config1": dict(p=dict(Nx=25, Ny=25, Nz=9, hx=0.5, hy=0.5, hz=0.5, kappa=2.0), B=(0.0, 0.0, 0.3)),
}


def build(td, case):
    """Build (device, params, idx, material) of one case with the reference."""
    p = td.SimulationParameters(**case["p"])
    tri = None
    if "trilayer" in case:
        b, i, t = case["trilayer"]
        tri = td.Trilayer(td.Layer(b[0], b[1], b[2]), td.Layer(i[0], i[1], i[2]), td.Layer(t[0], t[1], t[2]))
        p.Nz = tri.Nz
    bx, by, bz = case["B"]
    dev = td.Device(p, applied_field=td.AppliedField(Bx=bx, By=by, Bz=bz, t_on_fraction=1.0), trilayer=tri)
    for verts, zr in case.get("holes", []):
        dev.add_hole(verts, z_range=zr)
    if case.get("continuous"):
        rng = np.random.default_rng(7)
        from tdgl3d.core.material import MaterialMap
        kap = 1.5 + rng.random(p.dim_x)
        sc = rng.random(p.dim_x)
        dev._material = MaterialMap(kappa=kap, sc_mask=sc, interior_sc_mask=sc[dev.idx.interior_to_full])
    return dev


def random_state(params, seed):
    rng = np.random.default_rng(seed)
    n = params.n_interior
    nb = params.n_state // n
    psi = 0.7 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    phis = [0.5 * rng.standard_normal(n) for _ in range(nb - 1)]
    return np.concatenate([psi] + phis).astype(np.complex128)


def seeded_initial_state(dev, seed):
    """psi0 = initial_state + 0.01 (N + iN) * interior_sc_mask, phi0 = 0."""
    rng = np.random.default_rng(seed)
    x0 = dev.initial_state()
    n = dev.params.n_interior
    noise = 0.01 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    mask = dev.material.interior_sc_mask if dev.material is not None else 1.0
    x0.psi[:] += noise * mask
    return x0.data.copy()


def material_arrays(dev):
    m = dev.material
    if m is None:
        return {"has_material": np.array(0)}
    return {"has_material": np.array(1), "mat_kappa": m.kappa, "mat_sc": m.sc_mask,
            "mat_interior_sc": m.interior_sc_mask}


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print(f"  wrote {name}.npz ({os.path.getsize(path) / 1024:.1f} KiB)")


def case_meta(case):
    p = dict(case["p"])
    meta = {"p_" + k: np.array(v) for k, v in p.items()}
    meta["B"] = np.array(case["B"], dtype=np.float64)
    holes = case.get("holes", [])
    meta["n_holes"] = np.array(len(holes))
    for h, (verts, zr) in enumerate(holes):
        meta[f"hole{h}_vertices"] = np.array(verts, dtype=np.float64)
        meta[f"hole{h}_zrange"] = np.array(zr if zr is not None else (-1, -1))
    if "trilayer" in case:
        meta["trilayer"] = np.array([[a, b, float(c)] for a, b, c in case["trilayer"]], dtype=np.float64)
    meta["continuous"] = np.array(1 if case.get("continuous") else 0)
    return meta


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("TDGL3D_REFERENCE"),
                    help="checkout of omedeiro/nanowire_tdgl (its src/ is imported); or set TDGL3D_REFERENCE")
    ap.add_argument("--skip-long", action="store_true", help="skip the 101-step trajectory")
    args = ap.parse_args()
    if not args.reference:
        ap.error("--reference (or TDGL3D_REFERENCE) is required")
    sys.path.insert(0, os.path.join(args.reference, "src"))
    import tdgl3d as td
    from tdgl3d.physics.rhs import BoundaryVectors, eval_f
    from tdgl3d.physics.applied_field import build_boundary_field_vectors
    from tdgl3d.solvers.tgcr import tgcr_matrix_free_trap
    from tdgl3d.solvers.newton import newton_gcr_trap

    # ---- index maps, materials and eval_f on every case -------------------
    for name, case in CASES.items():
        dev = build(td, case)
        p, idx = dev.params, dev.idx
        arrs = {f"idx_{f}": np.asarray(getattr(idx, f)) for f in IDX_FIELDS}
        arrs.update(material_arrays(dev))
        arrs.update(case_meta(case))
        bx, by, bz = case["B"]
        u = BoundaryVectors(*build_boundary_field_vectors(bx, by, bz, p, idx))
        arrs["u_Bx"], arrs["u_By"], arrs["u_Bz"] = u.Bx, u.By, u.Bz
        X0 = seeded_initial_state(dev, seed=3)
        arrs["X_seeded"] = X0
        arrs["F_seeded"] = eval_f(X0, p, idx, u, material=dev.material)
        if name != "config1":   # keep the largest fixture small
            X = random_state(p, seed=11)
            arrs["X_random"] = X
            arrs["F_random"] = eval_f(X, p, idx, u, material=dev.material)
            # zero-field evaluation of the same random state
            u0 = BoundaryVectors(*build_boundary_field_vectors(0.0, 0.0, 0.0, p, idx))
            arrs["F_random_b0"] = eval_f(X, p, idx, u0, material=dev.material)
        save(f"case_{name}", **arrs)

    # ---- TGCR and Newton answers with the reference's own RHS --------------
    for name in ("3d_basic", "3d_hole", "2d_basic"):
        case = CASES[name]
        dev = build(td, case)
        p, idx = dev.params, dev.idx
        u = BoundaryVectors(*build_boundary_field_vectors(*case["B"], p, idx))
        calls = {"n": 0}

        def f(X):
            calls["n"] += 1
            return eval_f(X, p, idx, u, material=dev.material)

        x_lin = seeded_initial_state(dev, seed=5)
        rng = np.random.default_rng(9)
        b = 0.01 * random_state(p, seed=13)
        dt = 0.1
        calls["n"] = 0
        d = tgcr_matrix_free_trap(f, x_lin, b, dt, tol=1e-8, eps_mf=1e-4)
        k_tgcr = calls["n"] // 2
        fn = f(x_lin)
        x_pred = x_lin + dt * fn
        gamma = x_lin + dt / 2.0 * fn
        calls["n"] = 0
        xn, conv, iters = newton_gcr_trap(f, x_pred, gamma, dt, tol_f=1e-8, tol_dx=1e-3,
                                          max_iter=20, tol_gcr=1e-6, eps_mf=1e-4)
        save(f"solver_{name}", x_lin=x_lin, b=b, dt=np.array(dt), tgcr_tol=np.array(1e-8),
             tgcr_x=d, tgcr_iters=np.array(k_tgcr), x_pred=x_pred, gamma=gamma,
             newton_x=xn, newton_converged=np.array(int(conv)), newton_iters=np.array(iters),
             newton_f_calls=np.array(calls["n"]), rng_unused=np.array(rng.integers(1)))

    # ---- trajectories ------------------------------------------------------
    def run(name, t_stop, dt, method="trapezoidal", saves=None, seed=3, **kw):
        case = CASES[name]
        dev = build(td, case)
        x0 = seeded_initial_state(dev, seed=seed)
        t0 = time.time()
        sol = td.solve(dev, t_start=0.0, t_stop=t_stop, dt=dt, method=method, x0=x0,
                       progress=False, log_metadata=False, **kw)
        el = time.time() - t0
        keep = np.arange(sol.states.shape[1]) if saves is None else np.asarray(saves)
        out = dict(x0=x0, times=sol.times, saved_steps=keep, states=sol.states[:, keep],
                   wall_s=np.array(el), t_stop=np.array(t_stop), dt=np.array(dt))
        out.update({"kw_" + k: np.array(v) for k, v in kw.items()})
        # observables of the final saved state, as Solution computes them
        psi2 = sol.psi_squared(-1)
        Bx, By, Bz = sol.bfield(-1)
        Jx, Jy, Jz = sol.supercurrent_density(-1)
        out.update(psi2=psi2, Bx=Bx, By=By, Bz=Bz, Jx=Jx, Jy=Jy, Jz=Jz)
        return out, el

    trap_kw = dict(newton_tol_f=1e-8, newton_tol_dx=1e-3, tol_gcr=1e-6, eps_mf=1e-4)
    for name, t_stop in (("3d_basic", 1.0), ("2d_periodic_xy", 1.0), ("3d_hole", 1.0),
                         ("trilayer_hole", 1.0), ("3d_periodic_yz", 0.5), ("3d_hole_edge", 0.5)):
        out, el = run(name, t_stop, 0.1, **trap_kw)
        print(f"trap {name}: {el:.1f}s")
        save(f"trap_{name}", **out)
    out, el = run("3d_hole", 0.5, 0.01, method="euler", saves=[0, 1, 10, 50])
    print(f"euler 3d_hole: {el:.1f}s")
    save("euler_3d_hole", **out)
    if not args.skip_long:
        out, el = run("config1", 10.0, 0.1, saves=[0, 1, 2, 10, 50, 101], **trap_kw)
        print(f"trap config1 (101 steps): {el:.1f}s")
        save("trap_config1", **out)


if __name__ == "__main__":
    main()
