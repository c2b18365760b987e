"""Whole iterations and converged solves on the device, through the C ABI,
against the CPU oracle and against the reference's converged answers
(golden vectors). Tolerances are the parity contract: converged u, v, p, k,
omega within 1e-9 relative L2 of the reference."""
import numpy as np
import pytest

import cfd_b200 as cb
from helpers import Case, golden, golden_mesh, rel_err, rel_l2
from oracle import port

pytestmark = pytest.mark.gpu

CASES = ["laminar_cgrid", "sst_cgrid", "sst_cambered"]
CONVERGED_TOL = 1e-9


@pytest.mark.parametrize("name", CASES)
def test_twenty_iterations_track_the_oracle(name):
    c = Case(name)
    o = c.oracle(port.DEVICE_ORDER)
    d = c.device()
    mo = o.iterate(20)
    last, hist = d.iterate(20, history=True)
    assert np.all(np.isfinite(hist))
    # monitors: same CG iteration counts to within one, residuals close
    assert np.max(np.abs(hist[:, 5] - mo[:, 5])) <= 1
    for field, fid in (("U", 0), ("V", 1), ("P", 2), ("MASS_FLUX", 5)):
        assert rel_err(d.read(field), o.read(fid)) < 1e-7, field
    if c.model == 2:
        for field, fid in (("K", 22), ("OMEGA", 23), ("MUT", 24)):
            assert rel_err(d.read(field), o.read(fid)) < 1e-7, field


@pytest.mark.parametrize("name", CASES)
def test_converged_fields_match_the_reference(name):
    c = Case(name)
    g = c.g
    d = c.device()
    tol = 1e-12 if c.model == 0 else 1e-11
    taken, mon = d.converge(20000, tol)
    assert mon.worst() < tol, (taken, mon.worst())
    # settle k and omega as the golden state was settled
    mon = d.iterate(2000)
    assert mon.worst() < tol
    fields = [("U", "u"), ("V", "v"), ("P", "p")]
    if c.model == 2:
        fields += [("K", "k"), ("OMEGA", "omega"), ("MUT", "mut")]
    for field, key in fields:
        err = rel_l2(d.read(field), g[f"converged/{key}"])
        assert err < CONVERGED_TOL, (field, err)


def test_laminar_closure_is_bit_identical_to_no_closure():
    """TurbulenceTests.cpp:96-124: LaminarModel changes nothing."""
    c = Case("laminar_cgrid")
    a = c.device()
    b = cb.SimpleSolver.create(c.mesh, c.conditions, c.settings())
    b.set_turbulence_model(cb.MODEL_LAMINAR)
    b.initialise(*c.initial)
    a.iterate(15)
    b.iterate(15)
    for field in ("U", "V", "P", "MASS_FLUX", "MU_EFF"):
        assert np.array_equal(a.read(field), b.read(field)), field


def test_uniform_flow_is_reached_exactly():
    """ValidationTests.cpp:98-139 on the device: a wrong uniform start reaches
    the imposed stream to 1e-10 with max divergence < 1e-10."""
    g = golden("box_cases")
    mesh = cb.box(length=2.0, height=1.0, cells_x=20, cells_y=15, left=cb.FACE_FARFIELD,
                  right=cb.FACE_OUTLET, lower=cb.FACE_FARFIELD, upper=cb.FACE_FARFIELD)
    cond = cb.FaceConditions(g["uniform/kind"].astype(np.int32), g["uniform/velocity"],
                             g["uniform/pressure"])
    s = cb.SimpleSolver.create(mesh, cond, cb.Settings.defaults(velocity_relaxation=0.7,
                                                               pressure_relaxation=0.3))
    n = mesh.cells
    s.initialise(np.full(n, 0.4), np.zeros(n), np.zeros(n), np.ones(n), np.full(n, 0.05))
    taken, mon = s.converge(3000, 1e-12)
    assert taken < 3000
    assert np.max(np.abs(s.read("U") - 1.0)) < 1e-10
    assert np.max(np.abs(s.read("V"))) < 1e-10
    assert mon.max_divergence < 1e-10


def test_channel_matches_the_reference():
    """Plane channel (ValidationTests.cpp:203-275 set-up) against the
    reference's converged fields."""
    g = golden("box_cases")
    mesh = cb.box(length=4.0, height=1.0, cells_x=24, cells_y=16, grading=2,
                  first_cell_height=0.03)
    cond = cb.FaceConditions(g["channel/kind"].astype(np.int32), g["channel/velocity"],
                             g["channel/pressure"])
    s = cb.SimpleSolver.create(mesh, cond, cb.Settings.defaults(velocity_relaxation=0.7,
                                                               pressure_relaxation=0.3))
    n = mesh.cells
    s.initialise(np.ones(n), np.zeros(n), np.zeros(n), np.ones(n), np.full(n, 0.05))
    taken, mon = s.converge(6000, 1e-11)
    assert mon.worst() < 1e-11
    for field, key in (("U", "u"), ("V", "v"), ("P", "p")):
        assert rel_l2(s.read(field), g[f"channel/{key}"]) < CONVERGED_TOL, field


def test_divergence_and_mass_flux_accessors():
    c = Case("laminar_cgrid")
    d = c.device()
    d.iterate(3)
    o = c.oracle(port.DEVICE_ORDER)
    o.iterate(3)
    assert rel_err(d.divergence(), o.read(6)) < 1e-7
    assert d.mass_flux().shape == (c.mesh.faces,)


@pytest.mark.parametrize("name", CASES)
def test_forces_on_the_reference_field_match_the_reference(name):
    """extractSurface + integrateForces on the device, fed the reference's own
    converged field: Cl, Cd, Cm and every station's Cp as the reference's."""
    c = Case(name)
    g = c.g
    d = c.device()
    d.load_state(u=g["converged/u"], v=g["converged/v"], p=g["converged/p"],
                 mu_eff=g["converged/mu_eff"])
    f, cp, cf = d.forces(1.0, c.alpha, 1.0)
    ref = g["converged/forces"]
    for got, want in ((f.lift_coefficient, ref[0]), (f.drag_coefficient, ref[1]),
                      (f.moment_coefficient, ref[2]), (f.pressure_drag_coefficient, ref[3]),
                      (f.friction_drag_coefficient, ref[4])):
        assert got == pytest.approx(want, rel=1e-13, abs=1e-15)
    assert f.stations == int(ref[5])
    assert np.max(np.abs(cp - g["converged/cp"])) <= 1e-13 * max(1.0, np.max(np.abs(cp)))


@pytest.mark.parametrize("name", CASES)
def test_converged_forces_match_the_reference(name):
    """Cl, Cd and Cm of a converged device solve within 1e-7 relative of the
    reference's, and Cp at every station."""
    c = Case(name)
    g = c.g
    d = c.device()
    tol = 1e-12 if c.model == 0 else 1e-11
    d.converge(20000, tol)
    d.iterate(2000)
    f, cp, _ = d.forces(1.0, c.alpha, 1.0)
    ref = g["converged/forces"]
    assert f.lift_coefficient == pytest.approx(ref[0], rel=1e-7)
    assert f.drag_coefficient == pytest.approx(ref[1], rel=1e-7)
    assert f.moment_coefficient == pytest.approx(ref[2], rel=1e-7)
    assert np.max(np.abs(cp - g["converged/cp"])) < 1e-7


SEPARATION = ["laminar_a10", "laminar_a16", "sst_2412_a14"]


@pytest.mark.parametrize("name", SEPARATION)
def test_separation_points_match_the_reference(name):
    """findSeparation on the device (upper and lower surface, -1 where the
    layer stays attached) on the reference's own field at an incidence where
    it separates, with Cl/Cd/Cm and Cp as extractSurface/integrateForces give
    them (golden vectors from tests/golden/make_separation.py)."""
    g = golden("separation")
    sp, wp, npn, fl = g[f"{name}/grid"]
    des, alpha = str(g[f"{name}/designation"]), float(g[f"{name}/alpha"])
    mesh = cb.cgrid(des, surface_points=int(sp), wake_points=int(wp), normal_points=int(npn),
                    first_layer_height=float(fl), upstream_chords=10.0, downstream_chords=15.0,
                    vertical_chords=10.0)
    d = cb.SimpleSolver.create(mesh, cb.freestream_conditions(mesh, 1.0, alpha), cb.Settings.defaults())
    d.initialise(*cb.uniform_field(mesh, 1.0, alpha, 1.0, 1e6))
    d.load_state(u=g[f"{name}/u"], v=g[f"{name}/v"], p=g[f"{name}/p"], mu_eff=g[f"{name}/mu_eff"])
    f, cp, _ = d.forces(1.0, alpha, 1.0)
    ref = g[f"{name}/forces"]
    assert f.lift_coefficient == pytest.approx(ref[0], rel=1e-12)
    assert f.drag_coefficient == pytest.approx(ref[1], rel=1e-12)
    assert f.moment_coefficient == pytest.approx(ref[2], rel=1e-12, abs=1e-15)
    assert np.max(np.abs(cp - g[f"{name}/cp"])) <= 1e-12 * max(1.0, np.max(np.abs(cp)))
    assert f.separation_upper_chord_fraction == pytest.approx(ref[6], abs=1e-12)
    assert f.separation_lower_chord_fraction == pytest.approx(ref[7], abs=1e-12)
