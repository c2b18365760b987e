"""Python binding of the B200 SIMPLE solver's C ABI (include/cfd_gpu.h,
include/cfd_mesh.h), over ctypes.

The names mirror the reference's C++ interface so host code reads the same:
``SimpleSolver.create(mesh, conditions, settings)``, ``set_turbulence_model``,
``initialise``, ``iterate``, ``field``, ``mass_flux``, ``divergence``,
``set_settings`` (include/cfd/solver/SimpleSolver.hpp:159-274). Arrays are
numpy float64 in the reference's ordering (cells j*cellsI + i; faces j-faces
then i-faces; Vec2 arrays as (x, y) pairs).

The library is the in-tree ``libcfd_b200.so`` built by ``make`` in this
directory; importing this module fails loudly when it is missing. There is
no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libcfd_b200.so")

if not os.path.exists(LIBRARY_PATH):
    raise ImportError(
        f"{LIBRARY_PATH} is missing: build it with `make -C {_HERE}` (needs nvcc); "
        "the solver has no CPU fallback")
_lib = C.CDLL(LIBRARY_PATH)

# ---- status codes (ErrorCode + 1) --------------------------------------------
OK = 0
ERROR_NAMES = {1: "InvalidArgument", 2: "OutOfRange", 3: "NotFound", 4: "IoFailure",
               5: "NotImplemented", 6: "InitializationFailure", 7: "NumericalFailure",
               8: "Internal"}

BC_INTERNAL, BC_INLET, BC_OUTLET, BC_FARFIELD, BC_NOSLIP_WALL = range(5)
FACE_INTERIOR, FACE_WALL, FACE_FARFIELD, FACE_OUTLET, FACE_WAKECUT = range(5)

FIELDS = ["U", "V", "P", "RHO", "MU_EFF", "MASS_FLUX", "DIVERGENCE", "MU_MOLECULAR",
          "GRAD_U", "GRAD_V", "GRAD_P", "MOM_DIAG", "MOM_SOURCE_U", "MOM_SOURCE_V",
          "MOM_UPPER", "MOM_LOWER", "MOMENTUM_DIAGONAL", "P_DIAG", "P_SOURCE", "P_UPPER",
          "NET_FLUX", "P_CORRECTION", "K", "OMEGA", "MUT", "WALL_DISTANCE", "STRAIN", "F1",
          "F2", "CROSS_DIFFUSION", "PRODUCTION", "GRAD_K", "GRAD_OMEGA", "T_DIAG_K",
          "T_SOURCE_K", "T_DIAG_W", "T_SOURCE_W"]
FIELD = {name: k for k, name in enumerate(FIELDS)}
FACE_FIELDS = {"MASS_FLUX", "MOM_UPPER", "MOM_LOWER", "P_UPPER"}
VEC2_FIELDS = {"GRAD_U", "GRAD_V", "GRAD_P", "GRAD_K", "GRAD_OMEGA"}

STAGES = ["GRADIENTS", "MOMENTUM_ASSEMBLY", "MOMENTUM_SOLVE", "RHIE_CHOW",
          "PRESSURE_ASSEMBLY", "PRESSURE_SOLVE", "CORRECT", "SST_BLENDING", "SST_ASSEMBLY",
          "SST_SOLVE", "END"]
STAGE = {name: k for k, name in enumerate(STAGES)}

MODEL_NONE, MODEL_LAMINAR, MODEL_SST = 0, 1, 2


class CfdError(RuntimeError):
    """A non-zero cfd_status, with the library's message."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {message}")
        self.code = code


def _check(code: int) -> None:
    if code != OK:
        raise CfdError(code, _lib.cfd_last_error().decode())


# ---- C structs ------------------------------------------------------------------
class MeshDesc(C.Structure):
    _fields_ = [("nodes_i", C.c_int), ("nodes_j", C.c_int), ("cell_count", C.c_int),
                ("face_count", C.c_int), ("cell_centroids", C.c_void_p),
                ("cell_areas", C.c_void_p), ("face_centres", C.c_void_p),
                ("face_normals", C.c_void_p), ("face_areas", C.c_void_p),
                ("face_owner", C.c_void_p), ("face_neighbour", C.c_void_p),
                ("face_boundary", C.c_void_p), ("face_partner", C.c_void_p),
                ("nodes", C.c_void_p)]


class FaceBc(C.Structure):
    _fields_ = [("kind", C.c_void_p), ("velocity", C.c_void_p), ("pressure", C.c_void_p)]


class Settings(C.Structure):
    _fields_ = [("velocity_relaxation", C.c_double), ("pressure_relaxation", C.c_double),
                ("momentum_sweeps", C.c_int), ("pressure_iterations", C.c_int),
                ("pressure_tolerance", C.c_double), ("scheme", C.c_int),
                ("turbulence_relaxation", C.c_double), ("inflow_intensity", C.c_double),
                ("inflow_viscosity_ratio", C.c_double), ("inflow_length_scale", C.c_double),
                ("non_orthogonal_correctors", C.c_int), ("non_orthogonal_blend", C.c_double),
                ("precision", C.c_int), ("inner_iterations", C.c_int)]

    @staticmethod
    def defaults(**overrides) -> "Settings":
        s = Settings()
        _lib.cfd_default_settings(C.byref(s))
        for key, value in overrides.items():
            setattr(s, key, value)
        return s

    def packed(self) -> np.ndarray:
        """The 12-value layout the oracle and the reference harness take."""
        return np.array([self.velocity_relaxation, self.pressure_relaxation, self.momentum_sweeps,
                         self.pressure_iterations, self.pressure_tolerance, self.scheme,
                         self.turbulence_relaxation, self.inflow_intensity,
                         self.inflow_viscosity_ratio, self.inflow_length_scale,
                         self.non_orthogonal_correctors, self.non_orthogonal_blend], np.float64)


MONITOR_FIELDS = ["continuity", "momentum_x", "momentum_y", "mass_imbalance", "max_divergence",
                  "pressure_iterations", "turbulence_first", "turbulence_second", "min_energy",
                  "max_energy", "min_dissipation", "max_dissipation", "min_eddy_viscosity",
                  "max_eddy_viscosity", "max_eddy_viscosity_ratio", "max_wall_yplus"]


class Monitor(C.Structure):
    _fields_ = [("continuity", C.c_double), ("momentum_x", C.c_double),
                ("momentum_y", C.c_double), ("mass_imbalance", C.c_double),
                ("max_divergence", C.c_double), ("pressure_iterations", C.c_int),
                ("pad_", C.c_int), ("turbulence_first", C.c_double),
                ("turbulence_second", C.c_double), ("min_energy", C.c_double),
                ("max_energy", C.c_double), ("min_dissipation", C.c_double),
                ("max_dissipation", C.c_double), ("min_eddy_viscosity", C.c_double),
                ("max_eddy_viscosity", C.c_double), ("max_eddy_viscosity_ratio", C.c_double),
                ("max_wall_yplus", C.c_double)]

    def as_array(self) -> np.ndarray:
        return np.array([float(getattr(self, name)) for name in MONITOR_FIELDS])

    def worst(self) -> float:
        """ResidualSet::worst (FlowField.cpp:49-51)."""
        return max(abs(self.continuity), abs(self.momentum_x), abs(self.momentum_y))


class Forces(C.Structure):
    _fields_ = [("lift_coefficient", C.c_double), ("drag_coefficient", C.c_double),
                ("moment_coefficient", C.c_double), ("pressure_drag_coefficient", C.c_double),
                ("friction_drag_coefficient", C.c_double), ("lift", C.c_double),
                ("drag", C.c_double), ("pitching_moment", C.c_double),
                ("stagnation_chord_fraction", C.c_double), ("stations", C.c_int),
                ("leading_edge", C.c_int), ("separation_upper_chord_fraction", C.c_double),
                ("separation_lower_chord_fraction", C.c_double)]


class StreamlineOptions(C.Structure):
    _fields_ = [("max_steps", C.c_int), ("step_fraction", C.c_double), ("stall_fraction", C.c_double),
                ("reference_speed", C.c_double), ("trace_backwards", C.c_int)]


class CGridOptions(C.Structure):
    _fields_ = [("upstream_chords", C.c_double), ("downstream_chords", C.c_double),
                ("vertical_chords", C.c_double), ("surface_points", C.c_int),
                ("wake_points", C.c_int), ("normal_points", C.c_int),
                ("first_layer_height", C.c_double), ("normal_blend_length", C.c_double),
                ("normal_smoothing_passes", C.c_int)]


def _sig(name, restype, *argtypes):
    fn = getattr(_lib, name)
    fn.restype = restype
    fn.argtypes = list(argtypes)
    return fn


_P = C.c_void_p
_sig("cfd_last_error", C.c_char_p)
_sig("cfd_default_settings", None, _P)
_sig("cfd_set_device", C.c_int, C.c_int)
_sig("cfd_gpu_create", C.c_int, _P, _P, _P, _P)
_sig("cfd_gpu_set_turbulence", C.c_int, _P, C.c_int)
_sig("cfd_gpu_initialise", C.c_int, _P, _P, _P, _P, _P, _P)
_sig("cfd_gpu_iterate", C.c_int, _P, C.c_int, _P, _P)
_sig("cfd_gpu_converge", C.c_int, _P, C.c_int, C.c_double, _P, _P)
_sig("cfd_gpu_iterate_partial", C.c_int, _P, C.c_int, _P)
_sig("cfd_gpu_read_field", C.c_int, _P, C.c_int, _P)
_sig("cfd_gpu_load_state", C.c_int, _P, _P, _P, _P, _P, _P, _P, _P, _P)
_sig("cfd_gpu_set_settings", C.c_int, _P, _P)
_sig("cfd_gpu_forces", C.c_int, _P, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
     _P, _P, _P)
_sig("cfd_gpu_dims", C.c_int, _P, _P)
_sig("cfd_default_streamline_options", None, _P)
_sig("cfd_gpu_streamlines", C.c_int, _P, _P, C.c_int, _P, _P, _P, C.c_longlong, _P)
_sig("cfd_gpu_scalars", C.c_int, _P, _P)
_sig("cfd_gpu_destroy", C.c_int, _P)
_sig("cfd_default_cgrid_options", None, _P)
_sig("cfd_mesh_cgrid", C.c_int, C.c_char_p, _P, _P)
_sig("cfd_mesh_box", C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
     C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, _P)
_sig("cfd_mesh_describe", C.c_int, _P, _P)
_sig("cfd_mesh_nodes", _P, _P)
_sig("cfd_mesh_face_conditions", C.c_int, _P, C.c_double, C.c_double, _P, _P, _P)
_sig("cfd_mesh_free", None, _P)
_sig("cfd_cg_solve", C.c_int, _P, _P, C.c_double, C.c_int, _P, _P)
_sig("cfd_cg_solve_noalloc", C.c_int, _P, _P, C.c_double, C.c_int, _P, _P)
_sig("cfd_engine_create", C.c_int, C.c_ulonglong, C.c_int, _P)
_sig("cfd_engine_submit", C.c_int, _P, _P, _P)
_sig("cfd_engine_submit_sweep", C.c_int, _P, _P, C.c_double, C.c_double, C.c_double, C.c_int, _P, _P)
_sig("cfd_sweep_angles", C.c_int, C.c_double, C.c_double, C.c_double, _P, C.c_int, _P)
_sig("cfd_engine_step", C.c_int, _P, _P, _P)
_sig("cfd_engine_results", C.c_int, _P, _P, C.c_int, _P)
_sig("cfd_engine_surface", C.c_int, _P, C.c_int, _P, C.c_int, _P)
_sig("cfd_engine_set_shape_policy", C.c_int, _P, C.c_int)
_sig("cfd_engine_clock", C.c_double, _P)
_sig("cfd_engine_destroy", C.c_int, _P)
_sig("cfd_batch_create", C.c_int, _P, C.c_int, _P)
_sig("cfd_batch_iterate", C.c_int, _P, C.c_int, C.c_double, _P, _P)
_sig("cfd_batch_launch", C.c_int, _P, C.c_int, _P)
_sig("cfd_batch_graph_launch", C.c_int, _P, C.c_int, _P)
_sig("cfd_batch_monitors", C.c_int, _P, _P, _P)
_sig("cfd_batch_shape", C.c_int, _P, _P, _P)
_sig("cfd_batch_destroy", C.c_int, _P)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


# ---- meshes -----------------------------------------------------------------------
@dataclass
class MeshArrays:
    """A face-based structured mesh (cfd::mesh::Mesh's arrays)."""
    nodes_i: int
    nodes_j: int
    centroid: np.ndarray
    cell_area: np.ndarray
    face_centre: np.ndarray
    face_normal: np.ndarray
    face_area: np.ndarray
    owner: np.ndarray
    neighbour: np.ndarray
    boundary: np.ndarray
    partner: np.ndarray
    nodes: np.ndarray | None = None

    @property
    def cells(self) -> int:
        return int(self.cell_area.size)

    @property
    def faces(self) -> int:
        return int(self.face_area.size)

    @property
    def cells_i(self) -> int:
        return self.nodes_i - 1

    @property
    def cells_j(self) -> int:
        return self.nodes_j - 1

    def desc(self) -> MeshDesc:
        d = MeshDesc()
        d.nodes_i, d.nodes_j = self.nodes_i, self.nodes_j
        d.cell_count, d.face_count = self.cells, self.faces
        for name, arr in (("cell_centroids", self.centroid), ("cell_areas", self.cell_area),
                          ("face_centres", self.face_centre), ("face_normals", self.face_normal),
                          ("face_areas", self.face_area), ("face_owner", self.owner),
                          ("face_neighbour", self.neighbour), ("face_boundary", self.boundary),
                          ("face_partner", self.partner)):
            setattr(d, name, arr.ctypes.data)
        d.nodes = None if self.nodes is None else self.nodes.ctypes.data
        return d


def _take_mesh(handle: C.c_void_p) -> MeshArrays:
    d = MeshDesc()
    _check(_lib.cfd_mesh_describe(handle, C.byref(d)))
    n, f = d.cell_count, d.face_count

    def dbl(ptr, count):
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_double)), (count,)).copy()

    def i32(ptr, count):
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int)), (count,)).copy()

    nodes_ptr = _lib.cfd_mesh_nodes(handle)
    mesh = MeshArrays(d.nodes_i, d.nodes_j, dbl(d.cell_centroids, 2 * n), dbl(d.cell_areas, n),
                      dbl(d.face_centres, 2 * f), dbl(d.face_normals, 2 * f), dbl(d.face_areas, f),
                      i32(d.face_owner, f), i32(d.face_neighbour, f), i32(d.face_boundary, f),
                      i32(d.face_partner, f), dbl(nodes_ptr, 2 * d.nodes_i * d.nodes_j))
    return mesh


def default_cgrid_options(**overrides) -> CGridOptions:
    o = CGridOptions()
    _lib.cfd_default_cgrid_options(C.byref(o))
    for key, value in overrides.items():
        setattr(o, key, value)
    return o


def cgrid(designation: str, **options) -> MeshArrays:
    """generateCGrid for a closed-trailing-edge NACA section of chord 1."""
    opts = default_cgrid_options(**options)
    handle = C.c_void_p()
    _check(_lib.cfd_mesh_cgrid(designation.encode(), C.byref(opts), C.byref(handle)))
    try:
        return _take_mesh(handle)
    finally:
        _lib.cfd_mesh_free(handle)


def box(length=1.0, height=1.0, cells_x=40, cells_y=20, grading=0, first_cell_height=0.01,
        left=FACE_FARFIELD, right=FACE_OUTLET, lower=FACE_WALL, upper=FACE_WALL,
        origin_x=0.0, origin_y=0.0) -> MeshArrays:
    """generateBox (BoxGrid.cpp)."""
    handle = C.c_void_p()
    _check(_lib.cfd_mesh_box(origin_x, origin_y, length, height, cells_x, cells_y, grading,
                             first_cell_height, left, right, lower, upper, C.byref(handle)))
    try:
        return _take_mesh(handle)
    finally:
        _lib.cfd_mesh_free(handle)


@dataclass
class FaceConditions:
    kind: np.ndarray      # int32 per face
    velocity: np.ndarray  # 2 per face
    pressure: np.ndarray  # per face

    def struct(self) -> FaceBc:
        return FaceBc(self.kind.ctypes.data, self.velocity.ctypes.data, self.pressure.ctypes.data)


def freestream_velocity(speed: float, alpha_deg: float) -> tuple[float, float]:
    """FreestreamConditions::velocity (Freestream.cpp:11-14), with libm's cos/sin."""
    alpha = alpha_deg * math.pi / 180.0
    return speed * math.cos(alpha), speed * math.sin(alpha)


def freestream_conditions(mesh: MeshArrays, speed: float, alpha_deg: float) -> FaceConditions:
    """buildFaceConditions with the default BoundaryConditions
    (BoundaryConditions.cpp:73-97): wall -> no-slip, far field -> FarField,
    outlet -> Outlet, interior and wake cut -> Internal; pressure 0."""
    if not (math.isfinite(speed) and speed > 0):
        raise CfdError(1, "freestream speed must be positive")
    ux, uy = freestream_velocity(speed, alpha_deg)
    table = np.full(8, BC_INTERNAL, np.int32)
    table[FACE_WALL], table[FACE_FARFIELD], table[FACE_OUTLET] = BC_NOSLIP_WALL, BC_FARFIELD, BC_OUTLET
    kind = table[mesh.boundary].astype(np.int32)
    vel = np.zeros((mesh.faces, 2))
    vel[kind != BC_NOSLIP_WALL] = (ux, uy)
    return FaceConditions(kind, vel.reshape(-1).copy(), np.zeros(mesh.faces))


def uniform_field(mesh: MeshArrays, speed: float, alpha_deg: float, density: float,
                  reynolds: float, chord: float = 1.0):
    """FlowField::uniform (FlowField.cpp:21-47): (u, v, p, rho, mu)."""
    ux, uy = freestream_velocity(speed, alpha_deg)
    n = mesh.cells
    mu = density * speed * chord / reynolds
    return (np.full(n, ux), np.full(n, uy), np.zeros(n), np.full(n, density), np.full(n, mu))


# ---- solver ------------------------------------------------------------------------
class SimpleSolver:
    """A device-resident steady SIMPLE solve (SimpleSolver.hpp:159-274)."""

    def __init__(self, handle: C.c_void_p, mesh: MeshArrays):
        self._h = handle
        self.mesh = mesh

    @classmethod
    def create(cls, mesh: MeshArrays, conditions: FaceConditions,
               settings: Settings | None = None) -> "SimpleSolver":
        desc = mesh.desc()
        bc = conditions.struct()
        handle = C.c_void_p()
        _check(_lib.cfd_gpu_create(C.byref(desc), C.byref(bc),
                                   None if settings is None else C.byref(settings),
                                   C.byref(handle)))
        return cls(handle, mesh)

    def close(self) -> None:
        if self._h:
            _lib.cfd_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_turbulence_model(self, model: int) -> None:
        _check(_lib.cfd_gpu_set_turbulence(self._h, model))

    def initialise(self, u, v, p, rho, mu) -> None:
        arrays = [_f64(a) for a in (u, v, p, rho, mu)]
        _check(_lib.cfd_gpu_initialise(self._h, *[_ptr(a) for a in arrays]))

    def iterate(self, n: int = 1, history: bool = False):
        last = Monitor()
        hist = (Monitor * n)() if history else None
        _check(_lib.cfd_gpu_iterate(self._h, n, C.byref(last), hist))
        if history:
            return last, np.stack([h.as_array() for h in hist])
        return last

    def converge(self, cap: int, tol: float):
        last = Monitor()
        taken = C.c_int()
        _check(_lib.cfd_gpu_converge(self._h, cap, tol, C.byref(taken), C.byref(last)))
        return taken.value, last

    def iterate_partial(self, stage: str | int) -> Monitor:
        last = Monitor()
        code = STAGE[stage] if isinstance(stage, str) else stage
        _check(_lib.cfd_gpu_iterate_partial(self._h, code, C.byref(last)))
        return last

    def _size(self, name: str) -> int:
        n = self.mesh.cells
        return self.mesh.faces if name in FACE_FIELDS else (2 * n if name in VEC2_FIELDS else n)

    def read(self, name: str) -> np.ndarray:
        out = np.zeros(self._size(name))
        _check(_lib.cfd_gpu_read_field(self._h, FIELD[name], _ptr(out)))
        return out

    def read_into(self, name: str, out: np.ndarray) -> None:
        """read() into a caller's float64 buffer (e.g. pinned host memory)."""
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != self._size(name):
            raise ValueError(f"{name} needs a contiguous float64 buffer of {self._size(name)} values")
        _check(_lib.cfd_gpu_read_field(self._h, FIELD[name], _ptr(out)))

    def load_state(self, u=None, v=None, p=None, mass_flux=None, k=None, omega=None, mut=None,
                   mu_eff=None) -> None:
        arrays = [None if a is None else _f64(a) for a in (u, v, p, mass_flux, k, omega, mut, mu_eff)]
        _check(_lib.cfd_gpu_load_state(self._h, *[_ptr(a) for a in arrays]))

    def set_settings(self, settings: Settings) -> None:
        _check(_lib.cfd_gpu_set_settings(self._h, C.byref(settings)))

    def forces(self, speed: float, alpha_deg: float, density: float = 1.0,
               reference_pressure: float = 0.0, chord: float = 1.0):
        """extractSurface + integrateForces on the device: (Forces, Cp, Cf),
        stations upper (leading edge onwards) then lower."""
        f = Forces()
        cap = self.mesh.cells_i
        cp = np.zeros(cap)
        cf = np.zeros(cap)
        _check(_lib.cfd_gpu_forces(self._h, speed, alpha_deg, density, reference_pressure, chord,
                                   C.byref(f), _ptr(cp), _ptr(cf)))
        return f, cp[: f.stations], cf[: f.stations]

    def streamlines(self, seeds, max_steps: int = 4000, step_fraction: float = 0.35,
                    stall_fraction: float = 1e-4, reference_speed: float = 1.0,
                    trace_backwards: bool = True):
        """post::traceStreamlines on the device (cfd_gpu_streamlines): the
        point count per seed (0 where a seed is dropped) and the curves'
        points, one after another, as a (total, 2) array."""
        xy = np.ascontiguousarray(seeds, dtype=np.float64).reshape(-1, 2)
        n = xy.shape[0]
        o = StreamlineOptions()
        _lib.cfd_default_streamline_options(C.byref(o))
        o.max_steps, o.step_fraction, o.stall_fraction = max_steps, step_fraction, stall_fraction
        o.reference_speed, o.trace_backwards = reference_speed, 1 if trace_backwards else 0
        lengths = np.zeros(n, np.int32)
        total = C.c_longlong()
        _check(_lib.cfd_gpu_streamlines(self._h, _ptr(xy), n, C.byref(o), _ptr(lengths), None, 0,
                                        C.byref(total)))
        pts = np.zeros((max(total.value, 1), 2))
        _check(_lib.cfd_gpu_streamlines(self._h, _ptr(xy), n, C.byref(o), _ptr(lengths), _ptr(pts),
                                        total.value, C.byref(total)))
        return lengths, pts[: total.value]

    def scalars(self) -> np.ndarray:
        out = np.zeros(3)
        _check(_lib.cfd_gpu_scalars(self._h, _ptr(out)))
        return out

    # reference-style accessors
    def field(self) -> dict:
        return {name.lower(): self.read(name) for name in ("U", "V", "P", "RHO", "MU_EFF")}

    def mass_flux(self) -> np.ndarray:
        return self.read("MASS_FLUX")

    def divergence(self) -> np.ndarray:
        return self.read("DIVERGENCE")


class CgSystem(C.Structure):
    """cfd_cg_system: device pointers of a symmetric five-point LDU system."""
    _fields_ = [("cells_i", C.c_int), ("cells_j", C.c_int), ("diag", C.c_void_p),
                ("upper", C.c_void_p), ("source", C.c_void_p), ("across_j0", C.c_void_p)]


def cg_solve(system: CgSystem, x_ptr: int, tolerance: float, max_iterations: int,
             stream: int | None = None) -> np.ndarray:
    """conjugateGradient on the device (cfd_cg_solve); x_ptr is a device
    pointer to the start vector, overwritten with the solution. Returns the
    report {iterations, initial residual, final residual, converged}."""
    report = np.zeros(4)
    _check(_lib.cfd_cg_solve(C.byref(system), C.c_void_p(x_ptr), tolerance, max_iterations,
                             _ptr(report), None if stream is None else C.c_void_p(stream)))
    return report


def cg_solve_noalloc(system: CgSystem, x_ptr: int, tolerance: float, max_iterations: int,
                     stream: int | None = None) -> np.ndarray:
    """cfd_cg_solve without allocating: scratch is the library's fixed device
    array (blocks up to 65,536 nodes; calls must not overlap on the GPU)."""
    report = np.zeros(4)
    _check(_lib.cfd_cg_solve_noalloc(C.byref(system), C.c_void_p(x_ptr), tolerance,
                                     max_iterations, _ptr(report),
                                     None if stream is None else C.c_void_p(stream)))
    return report


def set_device(device: int) -> None:
    """Select the CUDA device later solves are created on (this thread)."""
    _check(_lib.cfd_set_device(device))


class Batch:
    """Many solves in one launch, one thread-block cluster each (cfd_batch_*)."""

    def __init__(self, solvers: list[SimpleSolver]):
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s._h for s in self.solvers])
        self._h = C.c_void_p()
        _check(_lib.cfd_batch_create(arr, len(self.solvers), C.byref(self._h)))

    def close(self) -> None:
        if self._h:
            _lib.cfd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def iterate(self, n: int, tol: float = -1.0):
        count = len(self.solvers)
        taken = (C.c_int * count)()
        last = (Monitor * count)()
        _check(_lib.cfd_batch_iterate(self._h, n, tol, taken, last))
        return list(taken), list(last)

    def launch(self, n: int, stream: int | None = None) -> None:
        """Enqueue n iterations on a CUDA stream (an int handle) without waiting."""
        _check(_lib.cfd_batch_launch(self._h, n, None if stream is None else C.c_void_p(stream)))

    def graph_launch(self, n: int, stream: int | None = None) -> None:
        """The same, replayed from a CUDA graph captured on first use."""
        _check(_lib.cfd_batch_graph_launch(self._h, n, None if stream is None else C.c_void_p(stream)))

    def monitors(self):
        count = len(self.solvers)
        taken = (C.c_int * count)()
        last = (Monitor * count)()
        _check(_lib.cfd_batch_monitors(self._h, taken, last))
        return list(taken), list(last)

    def shape(self) -> tuple[int, int]:
        cluster, threads = C.c_int(), C.c_int()
        _check(_lib.cfd_batch_shape(self._h, C.byref(cluster), C.byref(threads)))
        return cluster.value, threads.value


class Request(C.Structure):
    _fields_ = [("designation", C.c_char * 8), ("grid_surface_points", C.c_int),
                ("grid_wake_points", C.c_int), ("grid_normal_points", C.c_int),
                ("grid_first_layer_height", C.c_double), ("grid_upstream_chords", C.c_double),
                ("grid_downstream_chords", C.c_double), ("grid_vertical_chords", C.c_double),
                ("alpha_deg", C.c_double), ("reynolds", C.c_double), ("speed", C.c_double),
                ("density", C.c_double), ("model", C.c_int), ("tolerance", C.c_double),
                ("max_iterations", C.c_int), ("settings", Settings)]


class Result(C.Structure):
    _fields_ = [("id", C.c_int), ("status", C.c_int), ("iterations", C.c_int),
                ("retried_cold", C.c_int), ("cells", C.c_int), ("cluster_size", C.c_int),
                ("continuity", C.c_double), ("momentum_x", C.c_double),
                ("momentum_y", C.c_double), ("lift_coefficient", C.c_double),
                ("drag_coefficient", C.c_double), ("moment_coefficient", C.c_double),
                ("pressure_drag_coefficient", C.c_double),
                ("friction_drag_coefficient", C.c_double), ("submitted_s", C.c_double),
                ("started_s", C.c_double), ("finished_s", C.c_double),
                ("separation_upper_chord_fraction", C.c_double),
                ("separation_lower_chord_fraction", C.c_double), ("alpha_deg", C.c_double),
                ("continued", C.c_int), ("error", C.c_int), ("mesh_s", C.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


STATUS_NAMES = {0: "converged", 1: "iteration-limit", 2: "diverged", 3: "failed"}


def sweep_angles(start: float, end: float, step: float) -> list[float]:
    """post::sweepAngles (Polar.cpp:36-77) through the C ABI."""
    n = C.c_int()
    _check(_lib.cfd_sweep_angles(start, end, step, None, 0, C.byref(n)))
    out = np.zeros(max(n.value, 1))
    _check(_lib.cfd_sweep_angles(start, end, step, _ptr(out), n.value, C.byref(n)))
    return out[: n.value].tolist()


def request(designation: str, alpha_deg: float, reynolds: float, model: int = MODEL_SST,
            tolerance: float = 1e-6, max_iterations: int = 4000, surface_points: int = 128,
            wake_points: int = 65, normal_points: int = 97, first_layer_height: float = 1e-5,
            upstream_chords: float = 10.0, downstream_chords: float = 15.0,
            vertical_chords: float = 10.0, speed: float = 1.0, density: float = 1.0,
            settings: Settings | None = None) -> Request:
    r = Request()
    r.designation = designation.encode()[:8]
    r.grid_surface_points, r.grid_wake_points, r.grid_normal_points = surface_points, wake_points, normal_points
    r.grid_first_layer_height = first_layer_height
    r.grid_upstream_chords, r.grid_downstream_chords, r.grid_vertical_chords = (
        upstream_chords, downstream_chords, vertical_chords)
    r.alpha_deg, r.reynolds, r.speed, r.density = alpha_deg, reynolds, speed, density
    r.model, r.tolerance, r.max_iterations = model, tolerance, max_iterations
    r.settings = settings if settings is not None else Settings.defaults()
    return r


class Engine:
    """Continuous batching of many solves (cfd_engine_*)."""

    def __init__(self, memory_budget_bytes: int = 0, chunk: int = 32, tuned: bool = False):
        self._h = C.c_void_p()
        _check(_lib.cfd_engine_create(memory_budget_bytes, chunk, C.byref(self._h)))
        if tuned:
            _check(_lib.cfd_engine_set_shape_policy(self._h, 1))

    def close(self) -> None:
        if self._h:
            _lib.cfd_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, req: Request) -> int:
        out = C.c_int()
        _check(_lib.cfd_engine_submit(self._h, C.byref(req), C.byref(out)))
        return out.value

    def submit_sweep(self, base: Request, start: float, end: float, step: float,
                     continued: bool = True) -> list[int]:
        """A polar sweep run point after point (cfd_engine_submit_sweep): the
        ids of its points, in sweep order."""
        first, count = C.c_int(), C.c_int()
        _check(_lib.cfd_engine_submit_sweep(self._h, C.byref(base), start, end, step,
                                            1 if continued else 0, C.byref(first), C.byref(count)))
        return list(range(first.value, first.value + count.value))

    def step(self) -> tuple[int, int]:
        a, q = C.c_int(), C.c_int()
        _check(_lib.cfd_engine_step(self._h, C.byref(a), C.byref(q)))
        return a.value, q.value

    def results(self, capacity: int = 4096) -> list[Result]:
        buf = (Result * capacity)()
        count = C.c_int()
        _check(_lib.cfd_engine_results(self._h, buf, capacity, C.byref(count)))
        return [buf[k] for k in range(count.value)]

    def surface(self, request_id: int) -> np.ndarray:
        """Cp per wall station of a finished solve (taken once)."""
        n = C.c_int()
        _check(_lib.cfd_engine_surface(self._h, request_id, None, 0, C.byref(n)))
        cp = np.zeros(n.value)
        _check(_lib.cfd_engine_surface(self._h, request_id, _ptr(cp), n.value, C.byref(n)))
        return cp

    def clock(self) -> float:
        return float(_lib.cfd_engine_clock(self._h))

    def run(self, requests: list[Request]) -> list[Result]:
        """Submit everything, step until the engine is empty."""
        for r in requests:
            self.submit(r)
        return self.drain()

    def drain(self) -> list[Result]:
        """Step until every submitted request and sweep has finished."""
        out = []
        while True:
            active, queued = self.step()
            out.extend(self.results())
            if active == 0 and queued == 0:
                break
        out.extend(self.results())
        return sorted(out, key=lambda r: r.id)


def library_symbols() -> list[str]:
    """Names the C headers declare (for the ABI export check)."""
    return [name for name in dir(_lib) if name.startswith("cfd_")]


# ---- polar CSV ------------------------------------------------------------------------
def polar_csv(results, alphas=None, section: str = "", mesh: str = "", reynolds: float = 0.0,
              speed: float = 0.0, chord: float = 1.0, moment_reference: float = 0.25,
              continued_between_points: bool = False) -> str:
    """A polar in the reference's CSV layout (post::toCsv, Polar.cpp:126-164),
    so engine results can be diffed against the reference's examples/*.csv:
    a commented header, then one row per solve in the order given. `results`
    are engine Results; `alphas` their angles of attack in degrees (None: each
    result's own alpha_deg). Separation is an empty field where the surface
    stayed attached; l_over_d is 0 where Cd is not positive or not finite
    (AerodynamicForces::liftToDrag, Forces.cpp:50-56)."""
    if alphas is None:
        alphas = [r.alpha_deg for r in results]
    lines = ["# cfd_simulator aerodynamic polar",
             f"# section,{section or 'unknown'}",
             f"# mesh,{mesh or 'unknown'}",
             f"# reynolds,{reynolds:.6g}",
             f"# freestream_speed_mps,{speed:.6g}",
             f"# chord_m,{chord:.6g}",
             f"# moment_reference_xc,{moment_reference:.6g}",
             f"# continued_between_points,{'yes' if continued_between_points else 'no'}",
             "# every row is a separate Navier-Stokes solve; nothing is interpolated",
             "# status is converged, iteration-limit or diverged",
             "alpha_deg,cl,cd,cd_pressure,cd_friction,cm,l_over_d,"
             "separation_upper_xc,separation_lower_xc,status,iterations,continuity_residual"]
    for r, alpha in zip(results, alphas):
        cd = r.drag_coefficient
        l_over_d = r.lift_coefficient / cd if (math.isfinite(cd) and cd > 0.0) else 0.0
        upper = (f"{r.separation_upper_chord_fraction:.6f}"
                 if r.separation_upper_chord_fraction >= 0.0 else "")
        lower = (f"{r.separation_lower_chord_fraction:.6f}"
                 if r.separation_lower_chord_fraction >= 0.0 else "")
        # pointStatus: a point that never started has no converged flag set
        status = "diverged" if r.status == 2 else ("converged" if r.status == 0 else "iteration-limit")
        lines.append(f"{alpha:.6f},{r.lift_coefficient:.8f},{cd:.8f},"
                     f"{r.pressure_drag_coefficient:.8f},{r.friction_drag_coefficient:.8f},"
                     f"{r.moment_coefficient:.8f},{l_over_d:.6f},{upper},{lower},"
                     f"{status},{r.iterations},{r.continuity:.6e}")
    return "\n".join(lines) + "\n"
