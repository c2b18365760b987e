"""The C ABI library loads and exports every entry point include/*.h
declares; argument validation answers without touching a GPU."""
import ctypes
import os
import re

import pytest

import cfd_b200 as cb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for header in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not header.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", header)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(cfd_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_entry_point():
    lib = ctypes.CDLL(cb.LIBRARY_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_invalid_arguments_fail_with_codes():
    mesh = cb.box(cells_x=4, cells_y=3)
    cond = cb.freestream_conditions(mesh, 1.0, 0.0)
    with pytest.raises(cb.CfdError) as err:
        cb.SimpleSolver.create(mesh, cond, cb.Settings.defaults(velocity_relaxation=0.0))
    assert err.value.code == 1 and "relaxation" in str(err.value)
    with pytest.raises(cb.CfdError) as err:
        cb.SimpleSolver.create(mesh, cond, cb.Settings.defaults(pressure_relaxation=1.5))
    assert err.value.code == 1
    # a mesh whose counts do not match its structured block
    bad = cb.MeshArrays(mesh.nodes_i + 1, mesh.nodes_j, mesh.centroid, mesh.cell_area,
                        mesh.face_centre, mesh.face_normal, mesh.face_area, mesh.owner,
                        mesh.neighbour, mesh.boundary, mesh.partner)
    with pytest.raises(cb.CfdError) as err:
        cb.SimpleSolver.create(bad, cond, None)
    assert err.value.code == 1


def test_default_settings_are_the_reference_defaults():
    s = cb.Settings.defaults()
    assert (s.velocity_relaxation, s.pressure_relaxation, s.momentum_sweeps,
            s.pressure_iterations, s.pressure_tolerance, s.scheme, s.turbulence_relaxation,
            s.inflow_intensity, s.inflow_viscosity_ratio, s.inflow_length_scale,
            s.non_orthogonal_correctors, s.non_orthogonal_blend, s.precision) == (
        0.5, 0.2, 3, 200, 0.01, 0, 0.5, 0.001, 1.0, 0.0, 1, 1.0, 0)
