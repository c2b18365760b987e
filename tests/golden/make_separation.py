"""Golden separation points and force coefficients from the reference itself.

Run from the repository root where the reference sources are present:

    make -C oracle ref && python tests/golden/make_separation.py

For a few small C-grid cases at incidences where the boundary layer
separates, the reference's SimpleSolver runs from the uniform start
(iterate(), as its worker does), and its own extractSurface/integrateForces
(through oracle/reference.py) give Cl, Cd, Cm, Cp and the upper and lower
separation points (findSeparation). The final fields are stored with them, so
a test can load exactly that field into the device solver and compare its
surface data. Writes tests/golden/separation.npz.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import reference as R  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
DEFAULTS = np.array([0.5, 0.2, 3, 200, 0.01, 0, 0.5, 0.001, 1.0, 0.0, 1, 1.0])

CASES = {
    # name: (designation, surface, wake, normal, first layer, model, alpha, Re, iterations)
    "laminar_a10": ("0012", 24, 12, 13, 2e-3, 0, 10.0, 500.0, 3000),
    "laminar_a16": ("0012", 24, 12, 13, 2e-3, 0, 16.0, 500.0, 3000),
    "sst_2412_a14": ("2412", 24, 12, 13, 1e-4, 2, 14.0, 3e6, 1500),
}


def main() -> None:
    out = {}
    for name, (des, sp, wp, npn, fl, model, alpha, re, iters) in CASES.items():
        m = R.RefMesh.cgrid(des, sp, wp, npn, fl, 10.0, 15.0, 10.0)
        kind, vel, pres = m.conditions(1.0, alpha, 1.0, re)
        u, v, p, rho, mu = m.uniform(1.0, alpha, 1.0, re)
        settings = DEFAULTS.copy()
        settings[8] = 10.0
        s = R.RefSolver(m, kind, vel, pres, settings, turbulence=model)
        s.initialise(u, v, p, rho, mu)
        s.iterate(iters)
        forces, cp = s.forces(1.0, alpha, 1.0, re)
        out[f"{name}/grid"] = np.array([sp, wp, npn, fl])
        out[f"{name}/designation"] = np.array(des)
        out[f"{name}/alpha"] = np.array(alpha)
        out[f"{name}/u"] = s.read(R.U)
        out[f"{name}/v"] = s.read(R.V)
        out[f"{name}/p"] = s.read(R.P)
        out[f"{name}/mu_eff"] = s.read(R.MU_EFF)
        out[f"{name}/forces"] = forces
        out[f"{name}/cp"] = cp
        print(f"{name}: Cl {forces[0]:.5f} Cd {forces[1]:.5f} separation upper {forces[6]:.4f} "
              f"lower {forces[7]:.4f}")
    np.savez_compressed(os.path.join(OUT, "separation.npz"), **out)


if __name__ == "__main__":
    main()
