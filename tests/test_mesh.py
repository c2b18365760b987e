"""The library's own mesh generator against meshes the reference generated
(generateCGrid / generateBox -> buildStructured), bit for bit; plus the
validation the reference applies (CGrid.cpp:98-127, Naca4.cpp:23-63,
BoxGrid.cpp:7-22)."""
import numpy as np
import pytest

import cfd_b200 as cb
from helpers import golden_mesh

FIELDS = ("nodes", "centroid", "cell_area", "face_centre", "face_normal", "face_area", "owner",
          "neighbour", "boundary", "partner")


def _same(a: cb.MeshArrays, b: cb.MeshArrays):
    assert (a.nodes_i, a.nodes_j) == (b.nodes_i, b.nodes_j)
    for name in FIELDS:
        x, y = getattr(a, name), getattr(b, name)
        assert x.shape == y.shape, name
        assert np.array_equal(x, y), f"{name}: max |diff| {np.max(np.abs(x - y))}"


@pytest.mark.parametrize("name,designation,kw", [
    ("laminar_cgrid", "0012", dict(surface_points=24, wake_points=12, normal_points=13,
                                   first_layer_height=2e-3, upstream_chords=10.0,
                                   downstream_chords=15.0, vertical_chords=10.0)),
    ("sst_cgrid", "0012", dict(surface_points=24, wake_points=12, normal_points=13,
                               first_layer_height=1e-4, upstream_chords=10.0,
                               downstream_chords=15.0, vertical_chords=10.0)),
    ("sst_cambered", "2412", dict(surface_points=20, wake_points=8, normal_points=9,
                                  first_layer_height=5e-4)),
])
def test_cgrid_matches_reference_bitwise(name, designation, kw):
    _same(cb.cgrid(designation, **kw), golden_mesh(name))


def test_boxes_match_reference_bitwise():
    _same(cb.box(length=2.0, height=1.0, cells_x=12, cells_y=8, grading=1, first_cell_height=0.05,
                 left=cb.FACE_FARFIELD, right=cb.FACE_OUTLET, lower=cb.FACE_WALL,
                 upper=cb.FACE_FARFIELD), golden_mesh("box_graded"))
    _same(cb.box(length=1.0, height=1.0, cells_x=9, cells_y=7, grading=2, first_cell_height=0.04),
          golden_mesh("box_channel"))


def test_cgrid_topology():
    """C-grid facts the reference's CGridTests check: cellsI = 2*wake + 2*surface - 2,
    wake-cut partners pair face k with face ni-2-k, and cell areas are positive."""
    m = cb.cgrid("0012", surface_points=40, wake_points=20, normal_points=28)
    assert m.cells_i == 2 * 20 + 2 * 40 - 2
    assert m.cells_j == 27
    assert np.all(m.cell_area > 0.0)
    ni = m.nodes_i
    for k in range(m.cells_i):
        if m.boundary[k] == cb.FACE_WAKECUT:
            assert m.partner[k] == ni - 2 - k
            assert m.partner[m.partner[k]] == k
    # total wall faces: 2*surface - 2
    assert int(np.sum(m.boundary == cb.FACE_WALL)) == 2 * 40 - 2


@pytest.mark.parametrize("designation", ["12", "0412", "00120", "0000", "0041", "2x12", "0050"])
def test_bad_designations_are_rejected(designation):
    with pytest.raises(cb.CfdError) as err:
        cb.cgrid(designation, surface_points=16, wake_points=4, normal_points=5)
    assert err.value.code == 1


def test_bad_options_are_rejected():
    for kw in (dict(surface_points=7), dict(wake_points=1), dict(normal_points=2),
               dict(first_layer_height=0.0), dict(first_layer_height=0.2),
               dict(upstream_chords=0.5)):
        opts = dict(surface_points=16, wake_points=4, normal_points=5)
        opts.update(kw)
        with pytest.raises(cb.CfdError):
            cb.cgrid("0012", **opts)
    with pytest.raises(cb.CfdError):
        cb.box(cells_x=0)
    with pytest.raises(cb.CfdError):
        cb.box(grading=1, first_cell_height=0.5)
