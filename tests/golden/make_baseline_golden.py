"""Golden vectors at the benchmark grid sizes, generated by the reference itself.

Run from the repository root where the reference sources are present:

    make -C oracle ref && python tests/golden/make_baseline_golden.py

The three single-solve benchmark configurations:

  c1: NACA 0012, laminar, Re 500, alpha 0, C-grid 192 x 48 cells
      (surface 64, wake 33, normal 49 points), first layer 2e-3 chord
  c2: NACA 0012, k-omega SST, Re 1e6, alpha 4, intensity 0.1 %, mu_t/mu 10,
      C-grid 384 x 96 (128, 65, 97), first layer 1e-5
  c3: NACA 2412, k-omega SST, Re 3e6, alpha 6, intensity 0.1 %, mu_t/mu 10,
      C-grid 768 x 192 (256, 129, 193), first layer 5e-6

all with upstream and vertical extents of 10 chords and 15 downstream, the
SimpleSettings defaults and the uniform freestream start. For each it stores
what the reference's own code produced: SHA-256 digests of its mesh arrays,
the 20 monitors of its first 20 SimpleSolver::iterate() calls, and digests of
the fields after iterations 1 and 20 (and of the first pressure-correction
system). Digests pin the CPU oracle to the reference bit for bit at full size
without committing megabytes of fields. For c1 it also stores the converged
fields and forces (the SolverWorker stop rule at worst residual < 1e-12, then
2000 settling iterations), which the device solve is compared with.
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import reference as R  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "baseline_sizes.npz")

# SimpleSettings defaults in the 12-value packed layout, mu_t/mu per case.
DEFAULTS = np.array([0.5, 0.2, 3, 200, 0.01, 0, 0.5, 0.001, 1.0, 0.0, 1, 1.0])

CASES = {
    # name: (designation, surface, wake, normal, first layer, model, alpha, Re, mu_t/mu)
    "c1": ("0012", 64, 33, 49, 2e-3, 0, 0.0, 500.0, 1.0),
    "c2": ("0012", 128, 65, 97, 1e-5, 2, 4.0, 1e6, 10.0),
    "c3": ("2412", 256, 129, 193, 5e-6, 2, 6.0, 3e6, 10.0),
}
EXTENTS = (10.0, 15.0, 10.0)  # upstream, downstream, vertical chords
MESH_KEYS = ("nodes", "centroid", "cell_area", "face_centre", "face_normal", "face_area", "owner",
             "neighbour", "boundary", "partner")


def digest(a: np.ndarray) -> str:
    """SHA-256 of an array's values as little-endian float64 (int32 for index arrays)."""
    a = np.asarray(a)
    a = np.ascontiguousarray(a, "<i4" if a.dtype.kind in "iu" else "<f8")
    return hashlib.sha256(a.tobytes()).hexdigest()


def fields_of(s: R.RefSolver, model: int) -> dict:
    names = [("u", R.U), ("v", R.V), ("p", R.P), ("mass_flux", R.MASS_FLUX), ("mu_eff", R.MU_EFF)]
    if model == 2:
        names += [("k", R.K), ("omega", R.OMEGA), ("mut", R.MUT)]
    return {key: s.read(fid) for key, fid in names}


def make_case(name: str, out: dict) -> None:
    des, sp, wp, npn, fl, model, alpha, re, ratio = CASES[name]
    t0 = time.perf_counter()
    m = R.RefMesh.cgrid(des, sp, wp, npn, fl, *EXTENTS)
    settings = DEFAULTS.copy()
    settings[8] = ratio
    out[f"{name}/grid"] = np.array([sp, wp, npn, fl])
    out[f"{name}/designation"] = np.array(des)
    out[f"{name}/model"] = np.int32(model)
    out[f"{name}/alpha"] = alpha
    out[f"{name}/reynolds"] = re
    out[f"{name}/settings"] = settings
    out[f"{name}/cells"] = np.int32(m.cells)
    for key in MESH_KEYS:
        out[f"{name}/mesh_digest/{key}"] = np.array(digest(getattr(m, key)))
    kind, vel, pres = m.conditions(1.0, alpha, 1.0, re)
    init = m.uniform(1.0, alpha, 1.0, re)
    for key, a in (("kind", kind), ("bc_velocity", vel), ("bc_pressure", pres)):
        out[f"{name}/conditions_digest/{key}"] = np.array(digest(a))
    for key, a in zip(("u", "v", "p", "rho", "mu"), init):
        out[f"{name}/uniform_digest/{key}"] = np.array(digest(a))
    s = R.RefSolver(m, kind, vel, pres, settings, turbulence=model)
    s.initialise(*init)
    hist = [s.iterate(1)]
    for key, fid in (("p_diag", R.P_DIAG), ("p_source", R.P_SOURCE), ("p_upper", R.P_UPPER)):
        out[f"{name}/iter1_digest/{key}"] = np.array(digest(s.read(fid)))
    for key, a in fields_of(s, model).items():
        out[f"{name}/iter1_digest/{key}"] = np.array(digest(a))
    hist.append(s.iterate(19))
    out[f"{name}/history20"] = np.concatenate(hist)
    for key, a in fields_of(s, model).items():
        out[f"{name}/iter20_digest/{key}"] = np.array(digest(a))
    # a few sampled values, so a mismatch can be sized, not only detected
    idx = np.linspace(0, m.cells - 1, 64).astype(np.int64)
    out[f"{name}/sample_cells"] = idx
    for key, a in fields_of(s, model).items():
        if a.size == m.cells:
            out[f"{name}/iter20_sample/{key}"] = a[idx]
    print(f"{name}: {m.cells} cells, 20 iterations in {time.perf_counter() - t0:.1f} s, "
          f"last continuity {hist[-1][-1, 0]:.3e}", flush=True)


def make_c1_converged(out: dict) -> None:
    des, sp, wp, npn, fl, model, alpha, re, ratio = CASES["c1"]
    m = R.RefMesh.cgrid(des, sp, wp, npn, fl, *EXTENTS)
    settings = DEFAULTS.copy()
    settings[8] = ratio
    kind, vel, pres = m.conditions(1.0, alpha, 1.0, re)
    s = R.RefSolver(m, kind, vel, pres, settings, turbulence=model)
    s.initialise(*m.uniform(1.0, alpha, 1.0, re))
    t0 = time.perf_counter()
    taken, mon = s.converge(200000, 1e-12)
    settle = s.iterate(2000)
    f = fields_of(s, model)
    forces, cp = s.forces(1.0, alpha, 1.0, re)
    out["c1/converged/stop_rule_iterations"] = np.int32(taken)
    out["c1/converged/monitor"] = settle[-1]
    for key in ("u", "v", "p"):
        out[f"c1/converged/{key}"] = f[key]
    out["c1/converged/forces"] = forces
    out["c1/converged/cp"] = cp
    print(f"c1 converged: stop rule at {taken} iterations ({time.perf_counter() - t0:.0f} s), "
          f"worst {np.max(np.abs(mon[:3])):.2e}; Cl {forces[0]:.3e} Cd {forces[1]:.6f} "
          f"Cm {forces[2]:.3e}", flush=True)


if __name__ == "__main__":
    out: dict = {}
    for case in CASES:
        make_case(case, out)
    make_c1_converged(out)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({os.path.getsize(OUT) / 1e3:.0f} kB)")
