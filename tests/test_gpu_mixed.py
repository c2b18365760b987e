"""The mixed FP32/FP64 form (settings.precision = 1).

Assembly stays FP64 (bit-identical to the plain form). The momentum and
k/omega sweeps solve for FP32 corrections to the FP64 unknowns, and the
pressure correction is an FP32 flexible CG preconditioned by a multigrid
V-cycle inside an FP64 residual refinement, stopped by the reference's own
rule (sum |r| <= tolerance * sum |b|, LinearSystem.cpp:118-210). So the
pressure solve must meet the stopping rule on the FP64 system, and a
converged solve lands on the plain form's (and the reference's) fixed
point."""
import numpy as np
import pytest

import cfd_b200 as cb
from helpers import Case, rel_err, rel_l2
from oracle import port

pytestmark = pytest.mark.gpu

CASES = ["laminar_cgrid", "sst_cgrid", "sst_cambered"]
# The SST fixed point is not a zero of the k and omega systems (floors and the
# wall-cell omega act after the sweeps), so FP32 corrections keep rounding
# into it: observed 2e-8 relative L2 in k. The mixed form's contract is on
# the forces (delta Cl <= 1e-4); these bounds are 100x tighter.
MIXED_FIELD_TOL = 1e-6


def _l1_residual(c, d):
    diag, source, upper = d.read("P_DIAG"), d.read("P_SOURCE"), d.read("P_UPPER")
    x = d.read("P_CORRECTION")
    y = port.ldu_multiply(c.mesh, diag, upper, upper, x)
    return np.sum(np.abs(source - y)), np.sum(np.abs(source))


@pytest.mark.parametrize("warm", [0, 5])
@pytest.mark.parametrize("name", CASES)
def test_pressure_solve_meets_the_reference_stopping_rule(name, warm):
    # inner_iterations = 0: the multigrid CG may take up to pressure_iterations
    c = Case(name)
    s = c.settings(precision=1)
    s.inner_iterations = 0
    d = cb.SimpleSolver.create(c.mesh, c.conditions, s)
    d.set_turbulence_model(c.model)
    d.initialise(*c.initial)
    if warm:
        d.iterate(warm)
    mon = d.iterate_partial("PRESSURE_SOLVE")
    res, b = _l1_residual(c, d)
    assert 0 < mon.pressure_iterations < 200
    assert res <= 0.01 * b * (1 + 1e-9), (res / b, mon.pressure_iterations)


def _pair_from(c, a):
    """A mixed-form solver loaded with the plain solver a's state."""
    b = c.device(precision=1)
    state = {k: a.read(f) for k, f in (("u", "U"), ("v", "V"), ("p", "P"),
                                       ("mass_flux", "MASS_FLUX"), ("mu_eff", "MU_EFF"))}
    if c.model == 2:
        state.update({k: a.read(f) for k, f in (("k", "K"), ("omega", "OMEGA"), ("mut", "MUT"))})
    b.load_state(**state)
    return b


@pytest.mark.parametrize("name", CASES)
def test_assembly_equals_the_plain_form_and_sweeps_round_like_fp32(name):
    """Assembly runs in FP64 in both forms (bit-identical); the momentum
    sweeps of the mixed form solve for an FP32 correction, so the velocities
    after them differ by FP32 rounding of a small correction."""
    c = Case(name)
    a = c.device(precision=0)
    a.iterate(3)
    b = _pair_from(c, a)
    a.iterate_partial("MOMENTUM_ASSEMBLY")
    b.iterate_partial("MOMENTUM_ASSEMBLY")
    for f in ("MOM_DIAG", "MOM_SOURCE_U", "MOM_SOURCE_V", "MOM_UPPER", "MOM_LOWER"):
        assert np.array_equal(a.read(f), b.read(f)), f
    a = c.device(precision=0)
    a.iterate(3)
    b = _pair_from(c, a)
    a.iterate_partial("MOMENTUM_SOLVE")
    b.iterate_partial("MOMENTUM_SOLVE")
    for f in ("U", "V"):
        assert rel_err(b.read(f), a.read(f)) < 1e-6, f


@pytest.mark.parametrize("name", CASES)
def test_converged_mixed_solve_reaches_the_reference_fixed_point(name):
    c = Case(name)
    g = c.g
    d = c.device(precision=1)
    tol = 1e-12 if c.model == 0 else 1e-11
    taken, mon = d.converge(20000, tol)
    assert mon.worst() < tol, (taken, mon.worst())
    d.iterate(2000)
    fields = [("U", "u"), ("V", "v"), ("P", "p")]
    if c.model == 2:
        fields += [("K", "k"), ("OMEGA", "omega"), ("MUT", "mut")]
    for field, key in fields:
        err = rel_l2(d.read(field), g[f"converged/{key}"])
        assert err < MIXED_FIELD_TOL, (field, err)
    f, cp, _ = d.forces(1.0, c.alpha, 1.0)
    ref = g["converged/forces"]
    assert f.lift_coefficient == pytest.approx(ref[0], rel=1e-6, abs=1e-9)
    assert f.drag_coefficient == pytest.approx(ref[1], rel=1e-6)
    assert f.moment_coefficient == pytest.approx(ref[2], rel=1e-6, abs=1e-9)
    assert np.max(np.abs(cp - g["converged/cp"])) < 1e-6


@pytest.mark.parametrize("name", CASES)
def test_default_inner_cap_bounds_the_pressure_solve(name):
    c = Case(name)
    d = c.device(precision=1)
    d.iterate(5)
    mon = d.iterate_partial("PRESSURE_SOLVE")
    res, b = _l1_residual(c, d)
    assert 0 < mon.pressure_iterations <= cb.Settings.defaults().inner_iterations
    assert res < 0.5 * b


def test_precision_is_fixed_at_create():
    c = Case("laminar_cgrid")
    d = c.device(precision=1)
    with pytest.raises(cb.CfdError):
        d.set_settings(c.settings(precision=0))


@pytest.mark.parametrize("ctas", [8, 16])
def test_mixed_form_gives_the_same_bits_every_run(ctas, monkeypatch):
    # A C-grid 70 cells around: halving it gives 35 columns, where cells
    # across the wake cut would share a red-black colour, so the multigrid
    # stops coarsening before that level (two partners updated in the same
    # half-sweep would read each other, and the bits would vary from run to
    # run). On 8 and 16 CTAs (most of them owning one row or none), repeated
    # solves, in one launch or in launches of one iteration, agree bit for bit.
    monkeypatch.setenv("CFD_CLUSTER_SIZE", str(ctas))
    mesh = cb.cgrid("0012", surface_points=24, wake_points=12, normal_points=13, first_layer_height=1e-4,
                    upstream_chords=10.0, downstream_chords=15.0, vertical_chords=10.0)
    settings = cb.Settings.defaults(inflow_viscosity_ratio=10.0, precision=1)
    runs = []
    for chunk in (100, 100, 100, 1):
        s = cb.SimpleSolver.create(mesh, cb.freestream_conditions(mesh, 1.0, 4.0), settings)
        s.set_turbulence_model(cb.MODEL_SST)
        s.initialise(*cb.uniform_field(mesh, 1.0, 4.0, 1.0, 1e6))
        for _ in range(100 // chunk):
            s.iterate(chunk)
        runs.append(np.concatenate([s.read(f) for f in ("U", "V", "P", "K", "OMEGA")]))
        s.close()
    for r in runs[1:]:
        assert np.array_equal(r, runs[0])
