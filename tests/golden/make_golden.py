"""Generate the golden fixtures in this directory from the reference itself.

Run from the repository root where the reference sources are present:

    make -C oracle ref && python tests/golden/make_golden.py

It drives the reference's own code (oracle/_ref/libcfdref.so, compiled from
the reference sources by oracle/Makefile) through oracle/reference.py and
stores what it produced: meshes from generateCGrid/generateBox, monitors and
fields after whole SimpleSolver::iterate() calls, stage outputs the reference
keeps private, converged fields, LDU primitive results and force
coefficients. The tests compare the CPU restatement (oracle/) and the
library's mesh generator against these, and the device solver against them at
convergence. Inputs are small seeded synthetic cases (tiny C-grids and boxes).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import reference as R  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# SimpleSettings defaults, in the 12-value packed layout.
DEFAULTS = np.array([0.5, 0.2, 3, 200, 0.01, 0, 0.5, 0.001, 1.0, 0.0, 1, 1.0])
# cartesianSettings of tests/ValidationTests.cpp:62-67: alpha_u 0.7, alpha_p 0.3.
CARTESIAN = DEFAULTS.copy()
CARTESIAN[0], CARTESIAN[1] = 0.7, 0.3

CASES = {
    # name: (designation, surface, wake, normal, first layer, extents, model, alpha, Re, sst ratio)
    "laminar_cgrid": ("0012", 24, 12, 13, 2e-3, (10.0, 15.0, 10.0), 0, 4.0, 500.0, 1.0),
    "sst_cgrid": ("0012", 24, 12, 13, 1e-4, (10.0, 15.0, 10.0), 2, 4.0, 1e6, 10.0),
    "sst_cambered": ("2412", 20, 8, 9, 5e-4, (12.0, 25.0, 12.0), 2, 6.0, 3e6, 10.0),
}


def mesh_arrays(m: R.RefMesh) -> dict:
    return {"nodes_i": np.int32(m.nodes_i), "nodes_j": np.int32(m.nodes_j), "nodes": m.nodes,
            "centroid": m.centroid, "cell_area": m.cell_area, "face_centre": m.face_centre,
            "face_normal": m.face_normal, "face_area": m.face_area, "owner": m.owner,
            "neighbour": m.neighbour, "boundary": m.boundary, "partner": m.partner}


def make_meshes() -> None:
    out = {}
    for name, (des, sp, wp, npn, fl, ext, *_rest) in CASES.items():
        m = R.RefMesh.cgrid(des, sp, wp, npn, fl, *ext)
        for key, value in mesh_arrays(m).items():
            out[f"{name}/{key}"] = value
    # generateBox, graded towards the lower wall (flat-plate style)
    b = R.RefMesh.box(length=2.0, height=1.0, cells_x=12, cells_y=8, grading=1,
                      first_cell_height=0.05, left=2, right=3, lower=1, upper=2)
    for key, value in mesh_arrays(b).items():
        out[f"box_graded/{key}"] = value
    b2 = R.RefMesh.box(length=1.0, height=1.0, cells_x=9, cells_y=7, grading=2,
                       first_cell_height=0.04, left=2, right=3, lower=1, upper=1)
    for key, value in mesh_arrays(b2).items():
        out[f"box_channel/{key}"] = value
    np.savez_compressed(os.path.join(OUT, "meshes.npz"), **out)


def make_case(name: str) -> None:
    des, sp, wp, npn, fl, ext, model, alpha, re, ratio = CASES[name]
    m = R.RefMesh.cgrid(des, sp, wp, npn, fl, *ext)
    kind, vel, pres = m.conditions(1.0, alpha, 1.0, re)
    u, v, p, rho, mu = m.uniform(1.0, alpha, 1.0, re)
    settings = DEFAULTS.copy()
    settings[8] = ratio
    out = {"alpha": alpha, "reynolds": re, "model": model, "settings": settings, "kind": kind,
           "bc_velocity": vel, "bc_pressure": pres, "u0": u, "v0": v, "p0": p, "rho0": rho,
           "mu0": mu}

    # Stage outputs of the first iteration from the uniform start, through
    # the reference's own (private) stage functions.
    s = R.RefSolver(m, kind, vel, pres, settings, turbulence=model)
    s.initialise(u, v, p, rho, mu)
    out["init/mass_flux"] = s.read(R.MASS_FLUX)
    out["init/dead_band"] = s.read(R.DEAD_BAND)
    out["init/mu_eff"] = s.read(R.MU_EFF)
    out["init/reference_mass_flow"] = s.scalars()[0]
    out["geometry/diffusion"] = s.read(R.GEOM_DIFFUSION)
    out["geometry/weight"] = s.read(R.GEOM_WEIGHT)
    out["geometry/tangential"] = s.read(R.GEOM_TANGENTIAL)
    if model == 2:
        out["init/k"] = s.read(R.K)
        out["init/omega"] = s.read(R.OMEGA)
        out["init/mut"] = s.read(R.MUT)
        out["init/wall_distance"] = s.read(R.WALL_DISTANCE)
        out["init/sst_scalars"] = s.sst_scalars()[:2]
    s.stage(R.S_INTERPOLATE)
    s.stage(R.S_GRADIENTS)
    for key, fid in (("face_u", R.FACE_U), ("face_v", R.FACE_V), ("face_p", R.FACE_P),
                     ("grad_u", R.GRAD_U), ("grad_v", R.GRAD_V), ("grad_p", R.GRAD_P)):
        out[f"stage1/{key}"] = s.read(fid)
    s.stage(R.S_ASSEMBLE_U)
    s.stage(R.S_RELAX_U)
    out["stage1/mom_diag"] = s.read(R.MOM_DIAG)
    out["stage1/mom_source_u"] = s.read(R.MOM_SOURCE)
    out["stage1/mom_upper"] = s.read(R.MOM_UPPER)
    out["stage1/mom_lower"] = s.read(R.MOM_LOWER)
    s.stage(R.S_ASSEMBLE_V)
    s.stage(R.S_RELAX_V)
    out["stage1/mom_source_v"] = s.read(R.MOM_SOURCE)
    del s

    # Whole iterations: monitors and fields after 1 and after 5.
    s = R.RefSolver(m, kind, vel, pres, settings, turbulence=model)
    s.initialise(u, v, p, rho, mu)
    hist = [s.iterate(1)]
    out["iter1/p_diag"] = s.read(R.P_DIAG)
    out["iter1/p_source"] = s.read(R.P_SOURCE)
    out["iter1/p_upper"] = s.read(R.P_UPPER)
    out["iter1/p_lower"] = s.read(R.P_LOWER)
    out["iter1/net_flux"] = s.read(R.NET_FLUX)
    out["iter1/momentum_diagonal"] = s.read(R.MOMENTUM_DIAGONAL)
    fields = [("u", R.U), ("v", R.V), ("p", R.P), ("mass_flux", R.MASS_FLUX), ("mu_eff", R.MU_EFF)]
    sst_fields = [("k", R.K), ("omega", R.OMEGA), ("mut", R.MUT), ("strain", R.STRAIN),
                  ("f1", R.F1), ("f2", R.F2), ("cross_diffusion", R.CROSS_DIFFUSION),
                  ("production", R.PRODUCTION), ("grad_k", R.GRAD_K), ("grad_omega", R.GRAD_OMEGA)]
    for key, fid in fields + (sst_fields if model == 2 else []):
        out[f"iter1/{key}"] = s.read(fid)
    hist.append(s.iterate(4))
    out["history5"] = np.concatenate(hist)
    for key, fid in fields + (sst_fields[:3] if model == 2 else []):
        out[f"iter5/{key}"] = s.read(fid)
    del s

    # Converged: the SolverWorker stop rule at a tight tolerance, then 2000
    # more iterations. The stop rule reads only the flow residuals; k and
    # omega keep settling for a while after it fires, so the fixed point is
    # taken from the settled state.
    s = R.RefSolver(m, kind, vel, pres, settings, turbulence=model)
    s.initialise(u, v, p, rho, mu)
    taken, mon = s.converge(40000, 1e-12 if model == 0 else 1e-11)
    settle = s.iterate(2000)
    out["converged/stop_rule_iterations"] = np.int32(taken)
    out["converged/iterations"] = np.int32(taken + 2000)
    out["converged/monitor"] = settle[-1]
    for key, fid in fields + (sst_fields[:3] if model == 2 else []):
        out[f"converged/{key}"] = s.read(fid)
    forces, cp = s.forces(1.0, alpha, 1.0, re)
    out["converged/forces"] = forces
    out["converged/cp"] = cp
    print(f"{name}: {m.cells} cells, converged in {taken} iterations, worst "
          f"{max(abs(mon[0]), abs(mon[1]), abs(mon[2])):.2e}, Cl {forces[0]:.6f} Cd {forces[1]:.6f}")
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **out)


def make_linear_algebra() -> None:
    """LDU primitives on the first pressure-correction system of the laminar case."""
    des, sp, wp, npn, fl, ext, model, alpha, re, _ = CASES["laminar_cgrid"]
    m = R.RefMesh.cgrid(des, sp, wp, npn, fl, *ext)
    kind, vel, pres = m.conditions(1.0, alpha, 1.0, re)
    s = R.RefSolver(m, kind, vel, pres, DEFAULTS, 0)
    s.initialise(*m.uniform(1.0, alpha, 1.0, re))
    s.iterate(1)
    diag, src = s.read(R.P_DIAG), s.read(R.P_SOURCE)
    up, lo = s.read(R.P_UPPER), s.read(R.P_LOWER)
    mdiag = s.read(R.MOMENTUM_DIAGONAL)
    rng = np.random.default_rng(20261203)
    x = rng.standard_normal(m.cells)
    lib = R.lib()
    y = np.zeros(m.cells)
    lib.ref_ldu_multiply(m._h, R._p(diag), R._p(up), R._p(lo), R._p(x), R._p(y))
    # an asymmetric system with the momentum pattern for Gauss-Seidel
    asym_up = up * (1.0 + 0.3 * rng.random(up.size))
    asym_lo = lo * (1.0 + 0.3 * rng.random(lo.size))
    gs = x.copy()
    lib.ref_ldu_gauss_seidel(m._h, R._p(mdiag * 4.0), R._p(src), R._p(asym_up), R._p(asym_lo),
                             R._p(gs), 3)
    cg = np.zeros(m.cells)
    rep = np.zeros(4)
    lib.ref_ldu_cg(m._h, R._p(diag), R._p(src), R._p(up), R._p(lo), R._p(cg), 0.01, 200, R._p(rep))
    cg_tight = np.zeros(m.cells)
    rep_tight = np.zeros(4)
    lib.ref_ldu_cg(m._h, R._p(diag), R._p(src), R._p(up), R._p(lo), R._p(cg_tight), 1e-12, 2000,
                   R._p(rep_tight))
    fv = rng.standard_normal(m.faces)
    gg = np.zeros(2 * m.cells)
    lib.ref_green_gauss(m._h, R._p(fv), R._p(gg))
    np.savez_compressed(os.path.join(OUT, "linalg.npz"), diag=diag, source=src, upper=up, lower=lo,
                        x=x, spmv=y, gs_diag=mdiag * 4.0, gs_upper=asym_up, gs_lower=asym_lo,
                        gs=gs, cg=cg, cg_report=rep, cg_tight=cg_tight, cg_tight_report=rep_tight,
                        face_values=fv, green_gauss=gg)


def make_box_cases() -> None:
    """Cartesian validation cases of tests/ValidationTests.cpp, run by the reference."""
    out = {}
    # Uniform flow on a 20 x 15 box, every side an inlet but the outlet (:98-139).
    b = R.RefMesh.box(length=2.0, height=1.0, cells_x=20, cells_y=15, left=2, right=3, lower=2, upper=2)
    kind = np.zeros(b.faces, np.int32)
    vel = np.zeros(2 * b.faces)
    pres = np.zeros(b.faces)
    for f in range(b.faces):
        if b.boundary[f] == 0:
            continue
        if b.boundary[f] == 3:
            kind[f] = 2
        else:
            kind[f] = 1
            vel[2 * f] = 1.0
    s = R.RefSolver(b, kind, vel, pres, CARTESIAN, 0)
    n = b.cells
    s.initialise(np.full(n, 0.4), np.zeros(n), np.zeros(n), np.ones(n), np.full(n, 0.05))
    taken, mon = s.converge(3000, 1e-12)
    out.update({"uniform/kind": kind, "uniform/velocity": vel, "uniform/pressure": pres,
                "uniform/iterations": np.int32(taken), "uniform/monitor": mon,
                "uniform/u": s.read(R.U), "uniform/v": s.read(R.V), "uniform/p": s.read(R.P)})
    # Plane Poiseuille in a channel graded towards both walls (:203-275).
    b = R.RefMesh.box(length=4.0, height=1.0, cells_x=24, cells_y=16, grading=2,
                      first_cell_height=0.03, left=2, right=3, lower=1, upper=1)
    kind = np.zeros(b.faces, np.int32)
    vel = np.zeros(2 * b.faces)
    pres = np.zeros(b.faces)
    for f in range(b.faces):
        t = b.boundary[f]
        if t == 1:
            kind[f] = 4
        elif t == 2:
            kind[f] = 1
            vel[2 * f] = 1.0
        elif t == 3:
            kind[f] = 2
    n = b.cells
    s = R.RefSolver(b, kind, vel, pres, CARTESIAN, 0)
    s.initialise(np.ones(n), np.zeros(n), np.zeros(n), np.ones(n), np.full(n, 0.05))
    taken, mon = s.converge(6000, 1e-11)
    out.update({"channel/kind": kind, "channel/velocity": vel, "channel/pressure": pres,
                "channel/iterations": np.int32(taken), "channel/monitor": mon,
                "channel/u": s.read(R.U), "channel/v": s.read(R.V), "channel/p": s.read(R.P),
                "channel/mass_flux": s.read(R.MASS_FLUX)})
    print(f"box cases: uniform {out['uniform/iterations']} it, channel {out['channel/iterations']} it")
    np.savez_compressed(os.path.join(OUT, "box_cases.npz"), **out)


if __name__ == "__main__":
    make_meshes()
    for case in CASES:
        make_case(case)
    make_linear_algebra()
    make_box_cases()
