"""Shared helpers: golden fixtures as meshes and cases, and one driver that
runs the same case on the device solver and on the CPU oracle."""
from __future__ import annotations

import os

import numpy as np

import cfd_b200 as cb
from oracle import port

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def golden_mesh(name: str) -> cb.MeshArrays:
    g = golden("meshes")
    a = {k.split("/", 1)[1]: v for k, v in g.items() if k.startswith(name + "/")}
    return cb.MeshArrays(int(a["nodes_i"]), int(a["nodes_j"]), a["centroid"], a["cell_area"],
                         a["face_centre"], a["face_normal"], a["face_area"],
                         a["owner"].astype(np.int32), a["neighbour"].astype(np.int32),
                         a["boundary"].astype(np.int32), a["partner"].astype(np.int32),
                         a["nodes"])


class Case:
    """A golden C-grid case: mesh, conditions, settings, initial field."""

    def __init__(self, name: str):
        self.name = name
        self.g = golden(name)
        self.mesh = golden_mesh(name)
        g = self.g
        self.model = int(g["model"])
        self.alpha = float(g["alpha"])
        self.reynolds = float(g["reynolds"])
        self.conditions = cb.FaceConditions(g["kind"].astype(np.int32), g["bc_velocity"],
                                            g["bc_pressure"])
        self.packed = g["settings"]
        self.initial = (g["u0"], g["v0"], g["p0"], g["rho0"], g["mu0"])

    def settings(self, precision: int = 0) -> cb.Settings:
        p = self.packed
        return cb.Settings.defaults(precision=precision,
            velocity_relaxation=p[0], pressure_relaxation=p[1], momentum_sweeps=int(p[2]),
            pressure_iterations=int(p[3]), pressure_tolerance=p[4], scheme=int(p[5]),
            turbulence_relaxation=p[6], inflow_intensity=p[7], inflow_viscosity_ratio=p[8],
            inflow_length_scale=p[9], non_orthogonal_correctors=int(p[10]),
            non_orthogonal_blend=p[11])

    def oracle(self, gs_order=port.DEVICE_ORDER) -> port.OracleSolver:
        s = port.OracleSolver(self.mesh, self.conditions, self.packed, self.model, gs_order)
        s.initialise(*self.initial)
        return s

    def device(self, precision: int = 0) -> "cb.SimpleSolver":
        s = cb.SimpleSolver.create(self.mesh, self.conditions, self.settings(precision))
        s.set_turbulence_model(self.model)
        s.initialise(*self.initial)
        return s


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """max |a - b| / max(max |b|, tiny): an infinity-norm relative error."""
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) / scale


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
