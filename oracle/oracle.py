"""ctypes wrapper for the CPU oracle (test infrastructure only).

The oracle is a C restatement of the reference's coupled thermal LBM time step
(zzhao0930/MPI-Multi-Process-Version, natural-convection_{2,3}dim_*.f90); see
the header of ``lbm_oracle.c`` for the file:line map.  Only the tests, the
smoke check and bench.py's CPU-baseline leg use it, as the checker or as the
timed CPU restatement; the product path never loads it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblbm_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)


def build(force: bool = False) -> str:
    """Compile liblbm_oracle.so with the committed Makefile."""
    src = os.path.join(_HERE, "lbm_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liblbm_oracle.so"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.ora_grid_raw.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp]
        L.ora_mesh.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               _dp, _dp, _dp, _dp]
        L.ora_create.restype = ctypes.c_void_p
        L.ora_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.ora_set_macro.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.ora_set_macro_neq.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.ora_slope3.argtypes = [ctypes.c_double] * 6
        L.ora_slope3.restype = ctypes.c_double
        L.ora_destroy.argtypes = [ctypes.c_void_p]
        L.ora_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ora_check.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.ora_nusselt.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.ora_sums.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.ora_ptr.restype = _dp
        L.ora_ptr.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ora_params.argtypes = [ctypes.c_void_p, _dp]
        L.ora_itc.restype = ctypes.c_long
        L.ora_itc.argtypes = [ctypes.c_void_p]
        L.ora_interpolateF.restype = ctypes.c_double
        L.ora_interpolateF.argtypes = [ctypes.c_double] * 7
        L.ora_wall_gradient.restype = ctypes.c_double
        L.ora_wall_gradient.argtypes = [ctypes.c_double] * 6
        L.ora_cell_widths.argtypes = [_dp, ctypes.c_int, ctypes.c_double, _dp]
        L.ora_set_threads.argtypes = [ctypes.c_int]
        L.ora_get_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


GRID_KINDS = {"erf": 0, "tanh": 1, "uniform": 2}


def mesh(kind: str, stretch: float, nx: int, ny: int, nz: int = 0):
    """The reference's mesh() (2M:74-134): returns (x, y, z, dx0, length_LB, dt),
    coordinates 0..n+1 in lattice units."""
    x = np.zeros(nx + 2)
    y = np.zeros(ny + 2)
    z = np.zeros(nz + 2) if nz else None
    out = np.zeros(3)
    lib().ora_mesh(GRID_KINDS[kind], stretch, nx, ny, nz, _p(x), _p(y),
                   _p(z) if z is not None else None, _p(out))
    return x, y, z, float(out[0]), float(out[1]), float(out[2])


class Oracle:
    """One cavity on the CPU.  Field arrays are returned as (ny, nx) / (nz, ny, nx)
    views, populations as (..., Q)."""

    PTR = {"f": 0, "f_post": 1, "g": 2, "g_post": 3, "rho": 4, "u": 5, "v": 6, "w": 7,
           "T": 8, "F": 9, "x": 10, "y": 11, "z": 12}

    def __init__(self, dim, nx, ny, nz=1, x=None, y=None, z=None, dt=None, length_LB=None,
                 Ra=1e5, Pr=0.71, Ma=0.1, Thot=1.0, Tcold=0.0, grid="erf", stretch=3.2):
        if dim == 2:
            nz = 1
        if x is None:
            x, y, z, _, length_LB, dt = mesh(grid, stretch, nx, ny, nz if dim == 3 else 0)
        if z is None:
            z = np.zeros(nz + 2)
        self.dim, self.nx, self.ny, self.nz = dim, nx, ny, nz
        self.Q = 9 if dim == 2 else 19
        self.QT = 5 if dim == 2 else 7
        self._x, self._y, self._z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
        self.h = lib().ora_create(dim, nx, ny, nz, _p(self._x), _p(self._y), _p(self._z),
                                  float(dt), float(length_LB), float(Ra), float(Pr), float(Ma),
                                  float(Thot), float(Tcold))
        self.dt, self.length_LB = float(dt), float(length_LB)

    def __del__(self):
        if getattr(self, "h", None):
            lib().ora_destroy(self.h)
            self.h = None

    @property
    def shape(self):
        return (self.ny, self.nx) if self.dim == 2 else (self.nz, self.ny, self.nx)

    def _arr(self, name, count, extra=None):
        p = lib().ora_ptr(self.h, self.PTR[name])
        a = np.ctypeslib.as_array(p, shape=(count,))
        return a

    def field(self, name):
        n = self.nx * self.ny * self.nz
        return self._arr(name, n).reshape(self.shape).copy()

    def pops(self, name):
        n = self.nx * self.ny * self.nz
        q = self.Q if name in ("f", "f_post") else self.QT
        return self._arr(name, n * q).reshape(self.shape + (q,)).copy()

    def coords(self, axis):
        n = {"x": self.nx, "y": self.ny, "z": self.nz}[axis]
        return self._arr(axis, n + 2).copy()

    def set_macro(self, rho, u, v, w, T):
        arrs = [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (rho, u, v)]
        wa = np.ascontiguousarray(w, dtype=np.float64).ravel() if w is not None else None
        Ta = np.ascontiguousarray(T, dtype=np.float64).ravel()
        lib().ora_set_macro(self.h, _p(arrs[0]), _p(arrs[1]), _p(arrs[2]),
                            _p(wa) if wa is not None else None, _p(Ta))

    def set_macro_neq(self, rho, u, v, w, T):
        """Warm-start state: equilibrium plus the first-order non-equilibrium
        part from the fields' gradients (ora_set_macro_neq)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (rho, u, v)]
        wa = np.ascontiguousarray(w, dtype=np.float64).ravel() if w is not None else None
        Ta = np.ascontiguousarray(T, dtype=np.float64).ravel()
        lib().ora_set_macro_neq(self.h, _p(arrs[0]), _p(arrs[1]), _p(arrs[2]),
                                _p(wa) if wa is not None else None, _p(Ta))

    def step(self, n=1):
        lib().ora_step(self.h, int(n))

    @property
    def itc(self):
        return int(lib().ora_itc(self.h))

    def check(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        lib().ora_check(self.h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def nusselt(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        lib().ora_nusselt(self.h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def sums(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        lib().ora_sums(self.h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def params(self):
        out = np.zeros(9)
        lib().ora_params(self.h, _p(out))
        keys = ["viscosity_LB", "kappa", "gbeta", "tauf", "Snu", "Sq", "sig_k", "dt", "length_LB"]
        return dict(zip(keys, out.tolist()))


def interpolateF(x0, x1, x2, x, f0, f1, f2):
    return lib().ora_interpolateF(x0, x1, x2, x, f0, f1, f2)


def slope3(xa, qa, xm, qm, xb, qb):
    return lib().ora_slope3(xa, qa, xm, qm, xb, qb)


def set_threads(n: int):
    lib().ora_set_threads(int(n))


def get_threads() -> int:
    return int(lib().ora_get_threads())
