"""Shared pytest set-up: the ``gpu`` marker and golden-fixture helpers."""

from __future__ import annotations

import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden(name: str):
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name}.npz missing")
    return dict(np.load(path, allow_pickle=False))


def golden_names(prefix: str):
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def device_from_fixture(d):
    """Rebuild a Device of this package from a ``case_*`` fixture's metadata."""
    import nanowire_tdgl_b200 as tb

    pk = {k[2:]: d[k].item() for k in d if k.startswith("p_")}
    p = tb.SimulationParameters(**pk)
    tri = None
    if "trilayer" in d:
        rows = d["trilayer"]
        tri = tb.Trilayer(*(tb.Layer(int(r[0]), float(r[1]), bool(r[2])) for r in rows))
    bx, by, bz = (float(v) for v in d["B"])
    dev = tb.Device(p, applied_field=tb.AppliedField(Bx=bx, By=by, Bz=bz, t_on_fraction=1.0), trilayer=tri)
    for h in range(int(d["n_holes"])):
        verts = [tuple(v) for v in d[f"hole{h}_vertices"]]
        zr = tuple(int(v) for v in d[f"hole{h}_zrange"])
        dev.add_hole(verts, z_range=None if zr == (-1, -1) else zr)
    if int(d["continuous"]):
        # per-node kappa / sc are not derivable from the metadata: take them as given
        dev._material = tb.MaterialMap(kappa=d["mat_kappa"].copy(), sc_mask=d["mat_sc"].copy(),
                                       interior_sc_mask=d["mat_interior_sc"].copy())
    return dev
