"""Golden streamlines from the reference's own tracer: post::traceStreamlines
(src/post/Streamlines.cpp:80-197) run by the reference on fields its own
SimpleSolver produced.

Run from the repository root where the reference sources are present:

    make -C oracle ref && python tests/golden/make_streamlines_golden.py

Two laminar NACA 0012 cases (Re 500): the small 24/12/13 C-grid at alpha 4,
converged, and the 192x48 C-grid at alpha 0 after 300 iterations (a trace
needs a field, not a converged one). Seeds upstream, on both sides of the
wake cut, close to the section, in the far field and outside the domain; the
default options and a short one-way variant. Stores each case's u and v,
the seeds, and each seed's curve (or its drop).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import reference as R  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "streamlines.npz")
DEFAULTS = np.array([0.5, 0.2, 3, 200, 0.01, 0, 0.5, 0.001, 1.0, 0.0, 1, 1.0])
CASES = {
    # name: (surface, wake, normal, first layer, alpha, iterations or None to converge)
    "small": (24, 12, 13, 2e-3, 4.0, None),
    "c1": (64, 33, 49, 2e-3, 0.0, 300),
}
SEEDS = np.array([[-1.0, 0.2], [-1.0, -0.05], [-0.3, 0.001], [0.5, 0.08], [0.5, -0.08],
                  [1.2, 0.0005], [1.2, -0.0005], [3.0, 0.0], [6.0, 2.0], [-8.0, 5.0],
                  [100.0, 0.0], [0.3, 0.0]])
OPTIONS = {"default": dict(), "short": dict(max_steps=150, step_fraction=0.6, trace_backwards=False)}


def main() -> None:
    out = {"seeds": SEEDS}
    for name, (sp, wp, npn, fl, alpha, iters) in CASES.items():
        m = R.RefMesh.cgrid("0012", sp, wp, npn, fl, 10.0, 15.0, 10.0)
        kind, vel, pres = m.conditions(1.0, alpha, 1.0, 500.0)
        s = R.RefSolver(m, kind, vel, pres, DEFAULTS, 0)
        s.initialise(*m.uniform(1.0, alpha, 1.0, 500.0))
        if iters is None:
            s.converge(40000, 1e-10)
        else:
            s.iterate(iters)
        out[f"{name}/grid"] = np.array([sp, wp, npn, fl, alpha])
        out[f"{name}/u"] = s.read(R.U)
        out[f"{name}/v"] = s.read(R.V)
        for opt, kw in OPTIONS.items():
            lengths, pts = s.streamlines(SEEDS, **kw)
            out[f"{name}/{opt}/lengths"] = lengths
            out[f"{name}/{opt}/points"] = pts
            print(name, opt, lengths.tolist())
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({os.path.getsize(OUT) / 1e3:.0f} kB)")


if __name__ == "__main__":
    main()
