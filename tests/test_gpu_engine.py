"""The solve engine (continuous batching, cfd_engine_*): results alone and in
a mix are the same, results equal a direct solve, admission respects the
memory budget, and a diverging solve is retried cold once (Polar.cpp:109-121)
and then reported diverged."""
import os

import numpy as np
import pytest

import cfd_b200 as cb

pytestmark = pytest.mark.gpu

TINY = dict(surface_points=24, wake_points=12, normal_points=13, first_layer_height=1e-4)


def _req(designation="0012", alpha=4.0, re=1e6, model=cb.MODEL_SST, tol=1e-8, cap=3000, **kw):
    grid = dict(TINY)
    grid.update(kw.pop("grid", {}))
    return cb.request(designation, alpha, re, model=model, tolerance=tol, max_iterations=cap,
                      settings=cb.Settings.defaults(inflow_viscosity_ratio=10.0), **grid, **kw)


def _key(r):
    return (r.status, r.iterations, r.lift_coefficient, r.drag_coefficient, r.moment_coefficient)


def test_each_result_is_the_same_alone_and_in_the_mix():
    mix = [_req(alpha=4.0, tol=1e-6), _req("2412", alpha=6.0, re=3e6, tol=1e-6),
           _req(alpha=2.0, re=500.0, model=cb.MODEL_NONE, grid=dict(first_layer_height=2e-3)),
           _req("0015", alpha=-3.0, re=2e5, tol=1e-6,
                grid=dict(surface_points=20, wake_points=8, normal_points=9))]
    together = cb.Engine(chunk=16).run(mix)
    assert [r.id for r in together] == list(range(len(mix)))
    assert sum(r.status == 0 for r in together) >= 3
    for k, req in enumerate(mix):
        alone = cb.Engine(chunk=16).run([req])
        a, b = alone[0], together[k]
        assert a.status == b.status, (a.status, b.status)
        assert a.iterations == b.iterations
        for x, y in ((a.lift_coefficient, b.lift_coefficient), (a.drag_coefficient, b.drag_coefficient),
                     (a.moment_coefficient, b.moment_coefficient)):
            assert x == pytest.approx(y, rel=1e-12, abs=1e-15)


@pytest.mark.parametrize("precision", [0, 1])
def test_engine_result_equals_a_direct_solve(precision):
    settings = cb.Settings.defaults(inflow_viscosity_ratio=10.0, precision=precision)
    req = cb.request("0012", 4.0, 1e6, tolerance=1e-8, max_iterations=3000, settings=settings, **TINY)
    engine = cb.Engine(chunk=32)
    res = engine.run([req])[0]
    cp_engine = engine.surface(res.id)
    mesh = cb.cgrid("0012", upstream_chords=10.0, downstream_chords=15.0, vertical_chords=10.0,
                    **TINY)
    # the same launch shape as the engine's tuner chose (the reduction order
    # depends on the CTAs per solve)
    old = os.environ.get("CFD_CLUSTER_SIZE")
    os.environ["CFD_CLUSTER_SIZE"] = str(res.cluster_size)
    try:
        s = cb.SimpleSolver.create(mesh, cb.freestream_conditions(mesh, 1.0, 4.0), settings)
    finally:
        if old is None:
            os.environ.pop("CFD_CLUSTER_SIZE")
        else:
            os.environ["CFD_CLUSTER_SIZE"] = old
    s.set_turbulence_model(cb.MODEL_SST)
    s.initialise(*cb.uniform_field(mesh, 1.0, 4.0, 1.0, 1e6))
    taken, mon = s.converge(3000, 1e-8)
    f, cp, _ = s.forces(1.0, 4.0, 1.0)
    assert res.status == 0 and res.iterations == taken
    assert np.array_equal(cp_engine, cp)
    assert res.lift_coefficient == pytest.approx(f.lift_coefficient, rel=1e-12)
    assert res.drag_coefficient == pytest.approx(f.drag_coefficient, rel=1e-12)
    assert res.continuity == pytest.approx(mon.continuity, rel=1e-12)


def test_admission_by_memory_budget_runs_one_at_a_time():
    engine = cb.Engine(memory_budget_bytes=1, chunk=64)  # room for one resident solve
    for alpha in (0.0, 2.0, 4.0):
        engine.submit(_req(alpha=alpha, tol=1e-6))
    results, peak = [], 0
    while True:
        active, queued = engine.step()
        peak = max(peak, active)
        results.extend(engine.results())
        if active == 0 and queued == 0:
            break
    assert peak == 1
    assert sorted(r.id for r in results) == [0, 1, 2]
    assert all(r.status == 0 for r in results)
    starts = sorted(r.started_s for r in results)
    ends = sorted(r.finished_s for r in results)
    assert starts[1] >= ends[0] and starts[2] >= ends[1]


def test_a_diverging_solve_is_retried_cold_once_then_reported():
    bad = cb.Settings.defaults(velocity_relaxation=1.0, pressure_relaxation=1.0)
    req = cb.request("0012", 8.0, 1e6, model=cb.MODEL_NONE, tolerance=1e-8, max_iterations=2000,
                     settings=bad, **TINY)
    r = cb.Engine(chunk=16).run([req])[0]
    assert r.status == 2 and r.retried_cold == 1
    assert not np.isfinite(r.continuity) or not np.isfinite(r.momentum_x)


def test_iteration_limit_is_reported():
    r = cb.Engine(chunk=16).run([_req(tol=1e-30, cap=40)])[0]
    assert r.status == 1 and r.iterations == 40


def test_tuned_shape_is_fixed_per_grid_and_reported():
    reqs = [_req(alpha=a, tol=1e-5, cap=200) for a in (0.0, 2.0)]
    res = cb.Engine(chunk=32, tuned=True).run(reqs)
    shapes = {r.cluster_size for r in res}
    assert len(shapes) == 1 and shapes.pop() in (4, 8, 16)
    # the same grid in another tuned engine of the process: the same shape
    again = cb.Engine(chunk=32, tuned=True).run(reqs[:1])[0]
    assert again.cluster_size == res[0].cluster_size


def test_each_result_is_the_same_alone_and_in_the_mix_when_tuned():
    mix = [_req(alpha=4.0, tol=1e-6), _req("0015", alpha=-3.0, re=2e5, tol=1e-6,
                                            grid=dict(surface_points=20, wake_points=8, normal_points=9))]
    together = cb.Engine(chunk=16, tuned=True).run(mix)
    for k, req in enumerate(mix):
        a, b = cb.Engine(chunk=16, tuned=True).run([req])[0], together[k]
        assert (a.status, a.iterations, a.cluster_size) == (b.status, b.iterations, b.cluster_size)
        assert a.lift_coefficient == pytest.approx(b.lift_coefficient, rel=1e-12, abs=1e-15)


def _direct(mesh, alpha, cluster, start=None, tol=1e-8, cap=3000):
    """A solve run by hand on the engine's launch shape (its bits depend on
    the CTAs per solve), optionally from a given u, v, p."""
    old = os.environ.get("CFD_CLUSTER_SIZE")
    os.environ["CFD_CLUSTER_SIZE"] = str(cluster)
    try:
        s = cb.SimpleSolver.create(mesh, cb.freestream_conditions(mesh, 1.0, alpha),
                                   cb.Settings.defaults(inflow_viscosity_ratio=10.0))
    finally:
        if old is None:
            os.environ.pop("CFD_CLUSTER_SIZE")
        else:
            os.environ["CFD_CLUSTER_SIZE"] = old
    s.set_turbulence_model(cb.MODEL_SST)
    u, v, p, rho, mu = cb.uniform_field(mesh, 1.0, alpha, 1.0, 1e6)
    if start is not None:
        u, v, p = start  # FlowField::uniform, then velocity and pressure carried over
    s.initialise(u, v, p, rho, mu)
    taken, _ = s.converge(cap, tol)
    f, _, _ = s.forces(1.0, alpha, 1.0)
    return s, taken, f


def test_continued_sweep_is_the_reference_continuation():
    """A continued polar sweep (startPolarSweep / updatePolar, Panels.cpp:1601-1797):
    points in sweepAngles order, one after another, each after the first
    started from the previous point's final u and p with density, viscosity,
    k and omega from the freestream (Panels.cpp:1145-1156). The engine's
    points equal the same chain run by hand, bit for bit, whatever each
    point's outcome."""
    base = _req(alpha=0.0, tol=1e-8, cap=3000)
    engine = cb.Engine(chunk=32)
    ids = engine.submit_sweep(base, 0.0, 4.0, 2.0, continued=True)
    res = sorted(engine.drain(), key=lambda r: r.id)
    assert [r.id for r in res] == ids
    assert [r.alpha_deg for r in res] == [0.0, 2.0, 4.0]
    assert [r.continued for r in res] == [0, 1, 1]
    assert all(r.status in (0, 1) for r in res)  # converged or at the cap, not diverged
    mesh = cb.cgrid("0012", upstream_chords=10.0, downstream_chords=15.0, vertical_chords=10.0,
                    **TINY)
    start = None
    for r in res:
        s, taken, f = _direct(mesh, r.alpha_deg, r.cluster_size, start)
        assert r.iterations == taken
        assert r.lift_coefficient == pytest.approx(f.lift_coefficient, rel=1e-12, abs=1e-15)
        assert r.drag_coefficient == pytest.approx(f.drag_coefficient, rel=1e-12)
        start = (s.read("U"), s.read("V"), s.read("P"))
        s.close()
    # started cold, every point is the freestream solve; where both reach the
    # tolerance they reach the same fixed point
    cold = cb.Engine(chunk=32)
    cold.submit_sweep(base, 0.0, 4.0, 2.0, continued=False)
    rc = sorted(cold.drain(), key=lambda r: r.id)
    assert [r.continued for r in rc] == [0, 0, 0]
    assert rc[0].iterations == res[0].iterations
    for a, b in zip(res, rc):
        if a.status == 0 and b.status == 0:
            assert a.lift_coefficient == pytest.approx(b.lift_coefficient, abs=1e-5)


def test_descending_sweep_and_many_sweeps_share_the_engine():
    engine = cb.Engine(chunk=32)
    down = engine.submit_sweep(_req(alpha=0.0, tol=1e-6), 4.0, 0.0, 2.0)
    up = engine.submit_sweep(_req("2412", alpha=0.0, re=3e6, tol=1e-6), -2.0, 2.0, 2.0)
    single = engine.submit(_req(alpha=1.0, tol=1e-6))
    res = {r.id: r for r in engine.drain()}
    assert sorted(res) == sorted(down + up + [single])
    assert [res[i].alpha_deg for i in down] == [4.0, 2.0, 0.0]
    assert [res[i].alpha_deg for i in up] == [-2.0, 0.0, 2.0]
    assert res[single].continued == 0


def test_a_request_that_cannot_start_is_reported_failed_not_diverged():
    bad = _req(tol=1e-6)
    bad.settings.velocity_relaxation = 1.5  # refused by SimpleSolver::create (SimpleSolver.cpp:41-44)
    engine = cb.Engine(chunk=16)
    one = engine.submit(bad)
    sweep = engine.submit_sweep(bad, 0.0, 2.0, 1.0)
    res = {r.id: r for r in engine.drain()}
    for i in [one] + sweep:
        assert res[i].status == 3 and res[i].error == 1, (i, res[i].status, res[i].error)
    assert [res[i].alpha_deg for i in sweep] == [0.0, 1.0, 2.0]
