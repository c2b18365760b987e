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


def digest(a: np.ndarray) -> str:
    """SHA-256 of an array's values as little-endian float64 (int32 for index
    arrays): the form tests/golden/make_baseline_golden.py stores."""
    import hashlib
    a = np.asarray(a)
    a = np.ascontiguousarray(a, "<i4" if a.dtype.kind in "iu" else "<f8")
    return hashlib.sha256(a.tobytes()).hexdigest()


class BaselineCase:
    """A benchmark-size case (c1 192x48 laminar, c2 384x96 SST, c3 768x192
    SST) from tests/golden/baseline_sizes.npz, meshed by the library's own
    generator (pinned bit for bit to the reference's at these sizes)."""

    _golden = None

    def __init__(self, name: str):
        if BaselineCase._golden is None:
            BaselineCase._golden = golden("baseline_sizes")
        g = BaselineCase._golden
        self.name = name
        self.g = {k.split("/", 1)[1]: v for k, v in g.items() if k.startswith(name + "/")}
        sp, wp, npn, fl = self.g["grid"]
        self.designation = str(self.g["designation"])
        self.mesh = cb.cgrid(self.designation, surface_points=int(sp), wake_points=int(wp),
                             normal_points=int(npn), first_layer_height=float(fl),
                             upstream_chords=10.0, downstream_chords=15.0, vertical_chords=10.0)
        self.model = int(self.g["model"])
        self.alpha = float(self.g["alpha"])
        self.reynolds = float(self.g["reynolds"])
        self.packed = self.g["settings"]
        self.conditions = cb.freestream_conditions(self.mesh, 1.0, self.alpha)
        self.initial = cb.uniform_field(self.mesh, 1.0, self.alpha, 1.0, self.reynolds)

    def settings(self, precision: int = 0) -> cb.Settings:
        p = self.packed
        return cb.Settings.defaults(precision=precision, inflow_intensity=p[7],
                                    inflow_viscosity_ratio=p[8])

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
