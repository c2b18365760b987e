"""ctypes binding of the reference solver compiled from its own sources
(oracle/_ref/libcfdref.so, built by `make -C oracle ref`). Test
infrastructure: golden-vector generation and the CPU baseline only.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "_ref", "libcfdref.so")

# ref_solver_read identifiers (ref_harness.cpp RefField)
(U, V, P, RHO, MU_EFF, MASS_FLUX, DIVERGENCE, MU_MOL, FACE_U, FACE_V, FACE_P, GRAD_U, GRAD_V,
 GRAD_P, MOM_DIAG, MOM_SOURCE, MOM_UPPER, MOM_LOWER, MOMENTUM_DIAGONAL, P_DIAG, P_SOURCE,
 P_UPPER, P_LOWER, NET_FLUX, DEAD_BAND, GEOM_AREA, GEOM_DELTA, GEOM_TANGENTIAL, GEOM_DIFFUSION,
 GEOM_WEIGHT, K, OMEGA, MUT, WALL_DISTANCE, STRAIN, F1, F2, CROSS_DIFFUSION, PRODUCTION, GRAD_K,
 GRAD_OMEGA) = range(41)
FACE = {MASS_FLUX, FACE_U, FACE_V, FACE_P, MOM_UPPER, MOM_LOWER, P_UPPER, P_LOWER, DEAD_BAND,
        GEOM_DIFFUSION, GEOM_WEIGHT}
FACE2 = {GEOM_AREA, GEOM_DELTA, GEOM_TANGENTIAL}
CELL2 = {GRAD_U, GRAD_V, GRAD_P, GRAD_K, GRAD_OMEGA}

# ref_solver_stage identifiers
(S_INTERPOLATE, S_GRADIENTS, S_ASSEMBLE_U, S_ASSEMBLE_V, S_RELAX_U, S_RELAX_V, S_RHIE_CHOW,
 S_ASSEMBLE_PRESSURE, S_APPLY_EDDY, S_SST_STRAIN, S_SST_BLENDING, S_SST_TRANSPORT, S_SST_WALL,
 S_SST_EDDY, S_SST_RANGES) = range(15)

_lib = None


def available() -> bool:
    return os.path.exists(LIBRARY_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise ImportError(f"{LIBRARY_PATH} is missing (built only where the reference "
                              "sources are present: `make -C oracle ref`)")
        _lib = C.CDLL(LIBRARY_PATH)
        P_ = C.c_void_p
        d, i = C.c_double, C.c_int
        for name, res, args in [
            ("ref_last_error", C.c_char_p, []),
            ("ref_mesh_cgrid", P_, [C.c_char_p, i, i, i, d, d, d, d, d, i]),
            ("ref_mesh_box", P_, [d, d, d, d, i, i, i, d, i, i, i, i]),
            ("ref_mesh_free", None, [P_]),
            ("ref_mesh_counts", None, [P_, P_]),
            ("ref_mesh_arrays", None, [P_] * 11),
            ("ref_face_conditions", i, [P_, d, d, d, d, P_, P_, P_]),
            ("ref_uniform_field", i, [P_, d, d, d, d, d] + [P_] * 5),
            ("ref_solver_create", P_, [P_] * 5 + [i]),
            ("ref_solver_free", None, [P_]),
            ("ref_solver_initialise", i, [P_] * 6),
            ("ref_solver_iterate", None, [P_, i, P_, P_]),
            ("ref_solver_converge", i, [P_, i, d, P_]),
            ("ref_solver_read", i, [P_, i, P_]),
            ("ref_sst_scalars", i, [P_, P_]),
            ("ref_solver_scalars", None, [P_, P_]),
            ("ref_solver_stage", i, [P_, i]),
            ("ref_solver_correct", None, [P_, P_]),
            ("ref_solver_keep_momentum_diagonal", None, [P_]),
            ("ref_ldu_multiply", None, [P_] * 6),
            ("ref_ldu_gauss_seidel", None, [P_] * 6 + [i]),
            ("ref_ldu_cg", None, [P_] * 6 + [d, i, P_]),
            ("ref_green_gauss", None, [P_] * 3),
            ("ref_forces", i, [P_, d, d, d, d, d, P_, P_]),
            ("ref_sweep_angles", i, [d, d, d, P_, i]),
            ("ref_streamlines", C.c_longlong, [P_, P_, i, i, d, d, d, i, P_, P_, C.c_longlong]),
            ("ref_polar_csv", i, [C.c_char_p, C.c_char_p, d, d, d, d, i, i, P_, C.c_char_p, i]),
        ]:
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class RefMesh:
    """A mesh generated by the reference (generateCGrid / generateBox)."""

    def __init__(self, handle):
        if not handle:
            raise ValueError(lib().ref_last_error().decode())
        self._h = C.c_void_p(handle)
        counts = np.zeros(4, np.int32)
        lib().ref_mesh_counts(self._h, _p(counts))
        self.nodes_i, self.nodes_j, n, f = (int(x) for x in counts)
        self.nodes = np.zeros(2 * self.nodes_i * self.nodes_j)
        self.centroid = np.zeros(2 * n)
        self.cell_area = np.zeros(n)
        self.face_centre = np.zeros(2 * f)
        self.face_normal = np.zeros(2 * f)
        self.face_area = np.zeros(f)
        self.owner = np.zeros(f, np.int32)
        self.neighbour = np.zeros(f, np.int32)
        self.boundary = np.zeros(f, np.int32)
        self.partner = np.zeros(f, np.int32)
        lib().ref_mesh_arrays(self._h, _p(self.nodes), _p(self.centroid), _p(self.cell_area),
                              _p(self.face_centre), _p(self.face_normal), _p(self.face_area),
                              _p(self.owner), _p(self.neighbour), _p(self.boundary),
                              _p(self.partner))

    # the reference Mesh has no node accessor in ref_mesh_arrays' first slot;
    # it is filled from Mesh::nodes().

    @property
    def cells(self):
        return int(self.cell_area.size)

    @property
    def faces(self):
        return int(self.face_area.size)

    @classmethod
    def cgrid(cls, designation, surface_points=160, wake_points=56, normal_points=72,
              first_layer=3e-4, upstream=12.0, downstream=25.0, vertical=12.0, blend=0.06,
              smoothing=6):
        return cls(lib().ref_mesh_cgrid(designation.encode(), surface_points, wake_points,
                                        normal_points, first_layer, upstream, downstream,
                                        vertical, blend, smoothing))

    @classmethod
    def box(cls, length=1.0, height=1.0, cells_x=40, cells_y=20, grading=0,
            first_cell_height=0.01, left=2, right=3, lower=1, upper=1, origin_x=0.0,
            origin_y=0.0):
        return cls(lib().ref_mesh_box(origin_x, origin_y, length, height, cells_x, cells_y,
                                      grading, first_cell_height, left, right, lower, upper))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ref_mesh_free(self._h)
            self._h = None

    def conditions(self, speed, alpha_deg, density=1.0, reynolds=1e6):
        kind = np.zeros(self.faces, np.int32)
        vel = np.zeros(2 * self.faces)
        pres = np.zeros(self.faces)
        if lib().ref_face_conditions(self._h, speed, alpha_deg, density, reynolds, _p(kind),
                                     _p(vel), _p(pres)) != 0:
            raise ValueError(lib().ref_last_error().decode())
        return kind, vel, pres

    def uniform(self, speed, alpha_deg, density, reynolds, chord=1.0):
        out = [np.zeros(self.cells) for _ in range(5)]
        if lib().ref_uniform_field(self._h, speed, alpha_deg, density, reynolds, chord,
                                   *[_p(a) for a in out]) != 0:
            raise ValueError(lib().ref_last_error().decode())
        return out


class RefSolver:
    """The reference SimpleSolver (optionally with LaminarModel or KOmegaSST)."""

    def __init__(self, mesh: RefMesh, kind, velocity, pressure, settings_packed, turbulence=0):
        self.mesh = mesh
        self._keep = (np.ascontiguousarray(kind, np.int32), np.ascontiguousarray(velocity, np.float64),
                      np.ascontiguousarray(pressure, np.float64),
                      np.ascontiguousarray(settings_packed, np.float64))
        h = lib().ref_solver_create(mesh._h, *[_p(a) for a in self._keep], turbulence)
        if not h:
            raise ValueError(lib().ref_last_error().decode())
        self._h = C.c_void_p(h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ref_solver_free(self._h)
            self._h = None

    def initialise(self, u, v, p, rho, mu):
        arrays = [np.ascontiguousarray(a, np.float64) for a in (u, v, p, rho, mu)]
        if lib().ref_solver_initialise(self._h, *[_p(a) for a in arrays]) != 0:
            raise ValueError(lib().ref_last_error().decode())

    def iterate(self, n=1):
        hist = np.zeros((n, 15))
        lib().ref_solver_iterate(self._h, n, None, _p(hist))
        return hist

    def converge(self, cap, tol):
        mon = np.zeros(15)
        taken = lib().ref_solver_converge(self._h, cap, tol, _p(mon))
        return taken, mon

    def read(self, which):
        n, f = self.mesh.cells, self.mesh.faces
        size = f if which in FACE else 2 * f if which in FACE2 else 2 * n if which in CELL2 else n
        out = np.zeros(size)
        if lib().ref_solver_read(self._h, which, _p(out)) != 0:
            raise ValueError(lib().ref_last_error().decode())
        return out

    def stage(self, which):
        if lib().ref_solver_stage(self._h, which) != 0:
            raise ValueError(f"stage {which} unavailable")

    def correct(self, correction):
        lib().ref_solver_correct(self._h, _p(np.ascontiguousarray(correction, np.float64)))

    def keep_momentum_diagonal(self):
        lib().ref_solver_keep_momentum_diagonal(self._h)

    def streamlines(self, seeds, max_steps=4000, step_fraction=0.35, stall_fraction=1e-4,
                    reference_speed=1.0, trace_backwards=True):
        """post::traceStreamlines on the current field: (lengths per seed,
        points (total, 2)); a dropped seed has length 0."""
        xy = np.ascontiguousarray(seeds, dtype=np.float64).reshape(-1, 2)
        n = xy.shape[0]
        lengths = np.zeros(n, np.int32)
        args = (self._h, _p(xy), n, max_steps, step_fraction, stall_fraction, reference_speed,
                1 if trace_backwards else 0, _p(lengths))
        total = lib().ref_streamlines(*args, None, 0)
        if total < 0:
            raise ValueError(lib().ref_last_error().decode())
        pts = np.zeros((max(total, 1), 2))
        lib().ref_streamlines(*args, _p(pts), total)
        return lengths, pts[:total]

    def sst_scalars(self):
        out = np.zeros(5)
        lib().ref_sst_scalars(self._h, _p(out))
        return out

    def scalars(self):
        out = np.zeros(2)
        lib().ref_solver_scalars(self._h, _p(out))
        return out

    def forces(self, speed, alpha_deg, density, reynolds, chord=1.0):
        """(Cl, Cd, Cm, Cd_p, Cd_f, stations, upper and lower separation x/c or -1), Cp."""
        out = np.zeros(8)
        cp = np.zeros(4 * self.mesh.faces)
        if lib().ref_forces(self._h, speed, alpha_deg, density, reynolds, chord, _p(out), _p(cp)) != 0:
            raise ValueError(lib().ref_last_error().decode())
        return out, cp[: int(out[5])]


def sweep_angles(start, end, step):
    """post::sweepAngles: the list of angles, or ValueError with the
    reference's message."""
    n = lib().ref_sweep_angles(start, end, step, None, 0)
    if n < 0:
        raise ValueError(lib().ref_last_error().decode())
    out = np.zeros(max(n, 1))
    lib().ref_sweep_angles(start, end, step, _p(out), n)
    return out[:n].tolist()


def polar_csv(section, mesh, reynolds, speed, chord, moment_reference, continued, points):
    """post::toCsv of a polar; `points` is an (n, 13) array (see ref_polar_csv)."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 13)
    args = (section.encode(), mesh.encode(), reynolds, speed, chord, moment_reference,
            1 if continued else 0, pts.shape[0], _p(pts))
    n = lib().ref_polar_csv(*args, None, 0)
    buf = C.create_string_buffer(n + 1)
    lib().ref_polar_csv(*args, buf, n)
    return buf.raw[:n].decode()
