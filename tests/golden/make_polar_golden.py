"""Golden vectors for the polar driver's host-side semantics, produced by the
reference's own code: post::sweepAngles (src/post/Polar.cpp:36-77) on a set
of sweep requests (ascending, descending, a step that divides the range only
to rounding, a step that does not divide it, the 400-point cap, and the
refusals), and post::toCsv (Polar.cpp:126-164) on seeded polars.

Run from the repository root where the reference sources are present:

    make -C oracle ref && python tests/golden/make_polar_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import reference as R  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "polar.npz")

SWEEPS = [(0.0, 18.0, 2.0), (-4.0, 16.0, 1.0), (16.0, -4.0, 1.0), (0.0, 0.9, 0.3),
          (0.0, 1.0, 0.3), (1.0, 0.5, 0.2), (5.0, 5.0, 1.0), (0.0, 1e-10, 1.0),
          (-2.5, 12.25, 0.35), (0.0, 399.0, 1.0), (0.0, 400.0, 1.0), (0.0, 1.0, 0.0),
          (0.0, 1.0, -1.0), (float("nan"), 1.0, 1.0), (0.0, float("inf"), 1.0)]


def polar_points(seed: int, n: int) -> np.ndarray:
    """13 values per point: alpha, cl, cd, cd_p, cd_f, cm, l/d, upper and lower
    separation, converged, diverged, iterations, continuity residual."""
    rng = np.random.default_rng(seed)
    pts = np.zeros((n, 13))
    pts[:, 0] = np.round(rng.uniform(-5.0, 15.0, n), 3)
    pts[:, 1] = rng.normal(0.5, 0.6, n)
    pts[:, 2] = rng.uniform(0.005, 0.2, n)
    pts[:, 3] = pts[:, 2] * rng.uniform(0.2, 0.8, n)
    pts[:, 4] = pts[:, 2] - pts[:, 3]
    pts[:, 5] = rng.normal(-0.05, 0.05, n)
    pts[:, 7] = np.where(rng.random(n) < 0.5, rng.uniform(0.0, 1.0, n), -1.0)
    pts[:, 8] = np.where(rng.random(n) < 0.3, rng.uniform(0.0, 1.0, n), -1.0)
    status = rng.integers(0, 3, n)  # converged, iteration-limit, diverged
    pts[:, 9] = status == 0
    pts[:, 10] = status == 2
    pts[:, 11] = rng.integers(1, 20000, n)
    pts[:, 12] = 10.0 ** rng.uniform(-9.0, 1.0, n)
    # awkward values: Cd not positive, not finite, a negative zero, huge
    pts[0, 2], pts[1, 2] = 0.0, float("nan")
    pts[2, 1], pts[3, 1] = -0.0, 1.5e7
    pts[4, 12] = float("inf")
    with np.errstate(divide="ignore", invalid="ignore"):
        pts[:, 6] = np.where(np.isfinite(pts[:, 2]) & (pts[:, 2] > 0.0), pts[:, 1] / pts[:, 2], 0.0)
    return pts


CSVS = [("NACA 2412", "768x192", 3e6, 1.0, 1.0, 0.25, True, 101, 9),
        ("", "", 500.0, 50.0, 0.3, 0.25, False, 102, 6)]


def main() -> None:
    out = {}
    for k, (a, b, c) in enumerate(SWEEPS):
        out[f"sweep{k}/request"] = np.array([a, b, c])
        try:
            out[f"sweep{k}/angles"] = np.array(R.sweep_angles(a, b, c))
        except ValueError as e:
            out[f"sweep{k}/error"] = np.array(str(e))
    for k, (section, mesh, re, speed, chord, mref, cont, seed, n) in enumerate(CSVS):
        pts = polar_points(seed, n)
        out[f"csv{k}/points"] = pts
        out[f"csv{k}/header"] = np.array([section, mesh])
        out[f"csv{k}/numbers"] = np.array([re, speed, chord, mref, 1.0 if cont else 0.0])
        out[f"csv{k}/text"] = np.array(R.polar_csv(section, mesh, re, speed, chord, mref, cont, pts))
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
