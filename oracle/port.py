"""ctypes binding of the CPU restatement (cfd_oracle.c). Test infrastructure.

Mirrors the product binding's method names so a parity test can drive both
with the same code: ``create``, ``initialise``, ``iterate``, ``read``,
``load_state``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "_build", "liboracle.so")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY_PATH):
            raise ImportError(f"{LIBRARY_PATH} is missing: run `make -C {_HERE}`")
        _lib = C.CDLL(LIBRARY_PATH)
        P = C.c_void_p
        for name, res, args in [
            ("or_create", P, [P, P, P, P, P, C.c_int, C.c_int]),
            ("or_initialise", C.c_int, [P] * 6),
            ("or_iterate", C.c_int, [P, C.c_int, C.c_int, P]),
            ("or_read", C.c_int, [P, C.c_int, P]),
            ("or_load_state", None, [P] * 9),
            ("or_scalars", None, [P, P]),
            ("or_free", None, [P]),
            ("or_last_error", C.c_char_p, []),
            ("or_ldu_multiply", None, [P] * 6),
            ("or_ldu_gauss_seidel", None, [P] * 6 + [C.c_int, C.c_int]),
            ("or_ldu_cg", None, [P] * 6 + [C.c_double, C.c_int, P]),
            ("or_green_gauss", None, [P, P, P]),
        ]:
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


class OrMesh(C.Structure):
    _fields_ = [("nodes_i", C.c_int), ("nodes_j", C.c_int), ("cells", C.c_int),
                ("faces", C.c_int), ("centroid", C.c_void_p), ("cell_area", C.c_void_p),
                ("face_centre", C.c_void_p), ("face_normal", C.c_void_p),
                ("face_area", C.c_void_p), ("owner", C.c_void_p), ("neighbour", C.c_void_p),
                ("boundary", C.c_void_p), ("partner", C.c_void_p)]


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def mesh_struct(mesh) -> OrMesh:
    m = OrMesh()
    m.nodes_i, m.nodes_j, m.cells, m.faces = mesh.nodes_i, mesh.nodes_j, mesh.cells, mesh.faces
    for name in ("centroid", "cell_area", "face_centre", "face_normal", "face_area", "owner",
                 "neighbour", "boundary", "partner"):
        setattr(m, name, getattr(mesh, name).ctypes.data)
    return m


FACE_FIELDS = {5, 14, 15, 19}
VEC2_FIELDS = {8, 9, 10, 31, 32}

# Gauss-Seidel orders (bit 0: momentum red-black, bit 1: k and omega red-black)
LEXICOGRAPHIC = 0   # the reference
DEVICE_ORDER = 1    # the device solver: momentum red-black, k and omega lexicographic
RED_BLACK = 1       # for the LDU primitive: red-black
RED_BLACK_ALL = 3


class OracleSolver:
    """The restated SIMPLE solve, on a mesh held by the caller."""

    def __init__(self, mesh, conditions, settings_packed: np.ndarray, model: int = 0,
                 gs_order: int = DEVICE_ORDER):
        self.mesh = mesh
        self._m = mesh_struct(mesh)
        self._keep = (conditions.kind, conditions.velocity, conditions.pressure,
                      np.ascontiguousarray(settings_packed, dtype=np.float64))
        h = lib().or_create(C.byref(self._m), _p(self._keep[0]), _p(self._keep[1]),
                            _p(self._keep[2]), _p(self._keep[3]), model, gs_order)
        if not h:
            raise ValueError(lib().or_last_error().decode())
        self._h = C.c_void_p(h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_free(self._h)
            self._h = None

    def initialise(self, u, v, p, rho, mu):
        arrays = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, p, rho, mu)]
        if lib().or_initialise(self._h, *[_p(a) for a in arrays]) != 0:
            raise ValueError(lib().or_last_error().decode())

    def iterate(self, n: int = 1, stop_stage: int = 10) -> np.ndarray:
        mon = np.zeros((max(n, 1), 16))
        ran = lib().or_iterate(self._h, n, stop_stage, _p(mon))
        return mon[:ran]

    def read(self, which: int) -> np.ndarray:
        n = self.mesh.cells
        size = self.mesh.faces if which in FACE_FIELDS else (2 * n if which in VEC2_FIELDS else n)
        out = np.zeros(size)
        if lib().or_read(self._h, which, _p(out)) != 0:
            raise ValueError(f"unknown field {which}")
        return out

    def load_state(self, u=None, v=None, p=None, mass_flux=None, k=None, omega=None, mut=None,
                   mu_eff=None):
        arrays = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                  for a in (u, v, p, mass_flux, k, omega, mut, mu_eff)]
        lib().or_load_state(self._h, *[_p(a) for a in arrays])

    def scalars(self) -> np.ndarray:
        out = np.zeros(3)
        lib().or_scalars(self._h, _p(out))
        return out


def ldu_multiply(mesh, diag, upper, lower, x):
    m = mesh_struct(mesh)
    y = np.zeros(mesh.cells)
    lib().or_ldu_multiply(C.byref(m), _p(diag), _p(upper), _p(lower), _p(x), _p(y))
    return y


def ldu_gauss_seidel(mesh, diag, source, upper, lower, x, sweeps, order=LEXICOGRAPHIC):
    m = mesh_struct(mesh)
    x = np.array(x, dtype=np.float64)
    lib().or_ldu_gauss_seidel(C.byref(m), _p(diag), _p(source), _p(upper), _p(lower), _p(x),
                              sweeps, order)
    return x


def ldu_cg(mesh, diag, source, upper, lower, x, tol, max_iterations):
    m = mesh_struct(mesh)
    x = np.array(x, dtype=np.float64)
    rep = np.zeros(4)
    lib().or_ldu_cg(C.byref(m), _p(diag), _p(source), _p(upper), _p(lower), _p(x), tol,
                    max_iterations, _p(rep))
    return x, rep


def green_gauss(mesh, face_values):
    m = mesh_struct(mesh)
    out = np.zeros(2 * mesh.cells)
    lib().or_green_gauss(C.byref(m), _p(np.ascontiguousarray(face_values, dtype=np.float64)), _p(out))
    return out
