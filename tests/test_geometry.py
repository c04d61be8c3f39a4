"""Integer index maps, hole rasterisation and material maps: bit-exact
against the reference's own arrays (golden fixtures made from tdgl3d)."""

import numpy as np
import pytest

from conftest import device_from_fixture, golden, golden_names

from nanowire_tdgl_b200.geometry import (construct_indices, identify_boundary_links,
                                         identify_hole_nodes, point_in_polygon,
                                         SimulationParameters)

CASES = golden_names("case_")


@pytest.mark.parametrize("name", CASES)
def test_index_maps_bit_exact(name):
    d = golden(name)
    dev = device_from_fixture(d)
    for key in d:
        if not key.startswith("idx_"):
            continue
        mine = np.asarray(getattr(dev.idx, key[4:]))
        ref = d[key]
        assert mine.shape == ref.shape, key
        assert np.array_equal(mine.astype(np.int64), ref.astype(np.int64)), key


@pytest.mark.parametrize("name", CASES)
def test_material_bit_exact(name):
    d = golden(name)
    dev = device_from_fixture(d)
    if int(d["has_material"]) == 0:
        assert dev.material is None
        return
    m = dev.material
    assert np.array_equal(m.kappa, d["mat_kappa"])
    assert np.array_equal(m.sc_mask, d["mat_sc"])
    assert np.array_equal(m.interior_sc_mask, d["mat_interior_sc"])


def test_interior_order_k_fastest():
    # interior_to_full[:4] for Nx=4, Ny=5, Nz=4 (k fastest, i slowest)
    idx = construct_indices(SimulationParameters(Nx=4, Ny=5, Nz=4))
    assert list(idx.interior_to_full[:4]) == [36, 66, 96, 41]


def test_smallest_grid():
    idx = construct_indices(SimulationParameters(Nx=2, Ny=2, Nz=1))
    assert len(idx.interior_to_full) == 1


def test_point_in_polygon_cases():
    tri = [(0, 0), (10, 0), (5, 10)]
    assert point_in_polygon((5, 5), tri)
    assert not point_in_polygon((15, 5), tri)
    sq = [(0, 0), (4, 0), (4, 4), (0, 4)]
    # lower edge excluded (y > min), upper edge included (y <= max)
    assert not point_in_polygon((2, 0), sq)
    assert point_in_polygon((2, 4), sq)


def test_boundary_links_single_column():
    mask = np.zeros((11, 11, 6), dtype=bool)
    mask[5, 5, :] = True
    x = identify_boundary_links(mask, "x")
    assert len(x) == 2 * 6
    z = identify_boundary_links(mask, "z")
    assert len(z) == 0
    with pytest.raises(ValueError):
        identify_boundary_links(mask, "w")


def test_hole_nodes_shape_and_zrange():
    sq = [(5.0, 5.0), (15.0, 5.0), (15.0, 15.0), (5.0, 15.0)]
    m = identify_hole_nodes(sq, (0, 5), 1.0, 1.0, 20, 20, 10)
    assert m.shape == (21, 21, 11)
    assert m[10, 10, 5] and not m[10, 10, 6]


def test_parameter_validation():
    with pytest.raises(ValueError):
        SimulationParameters(Nx=1, Ny=4)
    with pytest.raises(ValueError):
        SimulationParameters(Nx=4, Ny=4, Nz=0)
