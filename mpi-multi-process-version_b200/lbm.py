"""Python host mirror of the reference's time-step interface over the C ABI.

The reference (zzhao0930/MPI-Multi-Process-Version) drives its step from
`program main` (natural-convection_2dim_mono.f90:283-380): mesh(), initial(),
then a `do while` loop over collision/streaming/boundary/macro subroutines with
check() every 2000 iterations, an MLUPS print and a Tecplot ASCII dump.  This
module keeps those names and meanings (`mesh`, `Cavity.initial`,
`Cavity.step`, `Cavity.check`, `run_main`, `output_ascii`) and calls the CUDA
library liblbm_b200.so through ctypes.  There is no CPU fallback: if the
library or a CUDA device is missing, the calls raise.
"""
from __future__ import annotations

import ctypes
import os
import time
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblbm_b200.so")

LBM_OK = 0
STORE = {"f64": 0, "f32": 1}  # 2 (binary16 storage) is retired: the library rejects it
MODE = {"fast": 0, "exact": 1}
GRID = {"erf": 0, "tanh": 1, "uniform": 2}

# every symbol include/lbm_b200.h declares
EXPORTS = [
    "lbm_abi_version", "lbm_error_string", "lbm_last_error", "lbm_mesh", "lbm_mesh_box", "lbm_derived_params",
    "lbm_create", "lbm_destroy", "lbm_init_reference", "lbm_init_equilibrium", "lbm_init_warm", "lbm_step", "lbm_run", "lbm_itc",
    "lbm_check", "lbm_nusselt", "lbm_sums", "lbm_get_macro", "lbm_set_macro", "lbm_get_populations",
    "lbm_set_populations", "lbm_synchronize", "lbm_stream", "lbm_device_bytes", "lbm_kernel_launches",
    "lbm_set_option", "lbm_get_option", "lbm_check_noalloc", "lbm_march_plan3d", "lbm_set_storage",
    "lbm_batch_create", "lbm_batch_destroy", "lbm_batch_size", "lbm_batch_cavity", "lbm_batch_init_reference",
    "lbm_batch_step", "lbm_batch_check", "lbm_batch_nusselt", "lbm_batch_run", "lbm_batch_run_masked", "lbm_batch_tune",
    "lbm_batch_set_option", "lbm_batch_get_option", "lbm_batch_synchronize", "lbm_batch_stream",
    "lbm_batch_set_storage", "lbm_batch_run_mixed",
    "lbm_create_slab", "lbm_halo_size", "lbm_halo_pack", "lbm_halo_unpack", "lbm_check_sums", "lbm_nusselt_sums",
]
BATCH_OPT = {"tile": 1, "nblocks": 2, "persistent": 3, "graphs": 4, "growth": 5, "storages": 6, "storage": 7,
             "pdl": 8}
OPT_KERNEL, OPT_NBLOCKS, OPT_L2PROMO, OPT_GRAPHS, OPT_RESIDENT = 1, 2, 3, 4, 5
OPT_TILEY, OPT_PLAN, OPT_WAIT_LIMIT, OPT_PDL = 6, 7, 8, 9
KERNELS = {"auto": 0, "direct": 1, "march": 2}


class LBMError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


class lbm_params(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32), ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("Ra", ctypes.c_double), ("Pr", ctypes.c_double), ("Ma", ctypes.c_double),
        ("Thot", ctypes.c_double), ("Tcold", ctypes.c_double),
        ("dt", ctypes.c_double), ("length_LB", ctypes.c_double),
        ("storage", ctypes.c_int32), ("mode", ctypes.c_int32), ("device", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


_dp = ctypes.POINTER(ctypes.c_double)
_lib = None


def lib():
    """Load liblbm_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run build.py (the CUDA path has no fallback)")
        L = ctypes.CDLL(LIB_PATH)
        L.lbm_error_string.restype = ctypes.c_char_p
        L.lbm_last_error.restype = ctypes.c_char_p
        L.lbm_mesh.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                               _dp, _dp, _dp, _dp, _dp, _dp]
        L.lbm_mesh_box.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp, _dp, _dp]
        L.lbm_derived_params.argtypes = [ctypes.POINTER(lbm_params), _dp]
        L.lbm_create.argtypes = [ctypes.POINTER(lbm_params), _dp, _dp, _dp, ctypes.POINTER(ctypes.c_void_p)]
        L.lbm_create_slab.argtypes = [ctypes.POINTER(lbm_params), _dp, _dp, _dp, ctypes.c_int32, ctypes.c_int32,
                                      ctypes.POINTER(ctypes.c_void_p)]
        L.lbm_halo_size.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]
        L.lbm_halo_pack.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]
        L.lbm_halo_unpack.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]
        L.lbm_check_sums.argtypes = [ctypes.c_void_p, _dp]
        L.lbm_nusselt_sums.argtypes = [ctypes.c_void_p, _dp]
        L.lbm_destroy.argtypes = [ctypes.c_void_p]
        L.lbm_init_reference.argtypes = [ctypes.c_void_p]
        L.lbm_init_equilibrium.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.lbm_init_warm.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.lbm_step.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        L.lbm_itc.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]
        L.lbm_run.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_double,
                              ctypes.POINTER(ctypes.c_int64), _dp, _dp]
        L.lbm_check.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.lbm_nusselt.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.lbm_sums.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.lbm_get_macro.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.lbm_set_macro.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.lbm_get_populations.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.lbm_set_populations.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.lbm_synchronize.argtypes = [ctypes.c_void_p]
        L.lbm_stream.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        L.lbm_device_bytes.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]
        L.lbm_kernel_launches.restype = ctypes.c_int64
        L.lbm_set_option.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64]
        L.lbm_get_option.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]
        L.lbm_check_noalloc.argtypes = [ctypes.c_void_p] * 8 + [ctypes.c_int64, _dp, _dp, ctypes.c_void_p]
        _pp = ctypes.POINTER(_dp)
        L.lbm_batch_create.argtypes = [ctypes.c_int32, ctypes.POINTER(lbm_params), _pp, _pp, _pp,
                                       ctypes.POINTER(ctypes.c_void_p)]
        L.lbm_batch_destroy.argtypes = [ctypes.c_void_p]
        L.lbm_batch_size.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]
        L.lbm_batch_cavity.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]
        L.lbm_batch_init_reference.argtypes = [ctypes.c_void_p]
        L.lbm_batch_step.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        L.lbm_batch_check.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.lbm_batch_nusselt.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.lbm_batch_run.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                    ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64)]
        L.lbm_batch_run_masked.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                           ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
        L.lbm_batch_tune.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                     ctypes.POINTER(ctypes.c_int32), _dp]
        L.lbm_batch_set_option.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64]
        L.lbm_batch_get_option.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]
        L.lbm_batch_synchronize.argtypes = [ctypes.c_void_p]
        L.lbm_batch_stream.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        L.lbm_batch_set_storage.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        L.lbm_batch_run_mixed.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p]
        L.lbm_set_storage.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        _lib = L
    return _lib


def _chk(status: int, where: str):
    if status != LBM_OK:
        raise LBMError(status, where, lib().lbm_last_error().decode())


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous, "need contiguous float64"
    return a.ctypes.data_as(_dp)


def kernel_launches() -> int:
    return int(lib().lbm_kernel_launches())


NOALLOC_MAX_NODES = 67108864


def check_noalloc(u, v, w, T, u_prev, v_prev, w_prev, T_prev, n, stream=0):
    """check() residuals on caller-owned device arrays, without any device
    allocation by the library (lbm_check_noalloc).  Arguments are device
    addresses (ints, e.g. a tensor's data_ptr()); w and w_prev are None in 2D.
    The previous-field arrays are overwritten with the current fields.
    Returns (errU, errT)."""
    a, b = ctypes.c_double(), ctypes.c_double()
    ptr = lambda x: None if x is None else ctypes.c_void_p(int(x))  # noqa: E731
    _chk(lib().lbm_check_noalloc(ptr(u), ptr(v), ptr(w), ptr(T), ptr(u_prev), ptr(v_prev), ptr(w_prev),
                                 ptr(T_prev), int(n), ctypes.byref(a), ctypes.byref(b),
                                 ctypes.c_void_p(int(stream)) if stream else None), "lbm_check_noalloc")
    return a.value, b.value


# ---------------------------------------------------------------------------
# mesh(): 2M:74-134 / 3M:122-189
# ---------------------------------------------------------------------------
@dataclass
class Mesh:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray | None
    dx0: float
    length_LB: float
    dt: float


def mesh(nx: int, ny: int, nz: int = 0, grid: str = "erf", stretch: float = 3.2) -> Mesh:
    """The reference's grid: erf-stretched (constA = 3.2) by default; tanh and
    uniform grids go through the same shift/scale (2M:94-116)."""
    x, y = np.zeros(nx + 2), np.zeros(ny + 2)
    z = np.zeros(nz + 2) if nz else None
    out = np.zeros(3)
    _chk(lib().lbm_mesh(GRID[grid], float(stretch), nx, ny, nz, _p(x), _p(y), _p(z),
                        _p(out[0:1]), _p(out[1:2]), _p(out[2:3])), "lbm_mesh")
    return Mesh(x, y, z, float(out[0]), float(out[1]), float(out[2]))


def mesh_box(nx: int, ny: int, nz: int = 0, lx: float = 1.0, ly: float = 1.0, lz: float = 1.0,
             grid: str = "tanh", stretch: float = 1.5) -> Mesh:
    """mesh() for a box of physical size lx x ly (x lz) with any node counts:
    the finest first cell over the axes sets the lattice unit (lbm_mesh_box).
    Equal to mesh() for the unit square/cube with equal node counts."""
    x, y = np.zeros(nx + 2), np.zeros(ny + 2)
    z = np.zeros(nz + 2) if nz else None
    out = np.zeros(3)
    _chk(lib().lbm_mesh_box(GRID[grid], float(stretch), nx, ny, nz, float(lx), float(ly), float(lz), _p(x), _p(y),
                            _p(z), _p(out[0:1]), _p(out[1:2]), _p(out[2:3])), "lbm_mesh_box")
    return Mesh(x, y, z, float(out[0]), float(out[1]), float(out[2]))


# ---------------------------------------------------------------------------
# one cavity
# ---------------------------------------------------------------------------
class Cavity:
    """A differentially heated cavity on one GPU.

    dim=2: D2Q9 MRT + D2Q5 (hot wall x = 1, cold wall x = nx, gravity along y);
    dim=3: D3Q19 MRT + D3Q7 (hot wall y = 1, cold wall y = ny, gravity along z),
    as in the reference.  Fields come back in the Fortran layout a(nx, ny[, nz])
    as numpy arrays of shape (ny, nx) / (nz, ny, nx) (C order, x fastest)."""

    def __init__(self, dim: int, nx: int, ny: int, nz: int = 1, Ra: float = 1e5, Pr: float = 0.71,
                 Ma: float = 0.1, Thot: float = 1.0, Tcold: float = 0.0, grid: str = "erf",
                 stretch: float = 3.2, storage: str = "f64", mode: str = "fast", device: int = 0,
                 coords: Mesh | None = None, kernel: str = "auto", nblocks: int = 0):
        if dim == 2:
            nz = 1
        m = coords or mesh(nx, ny, nz if dim == 3 else 0, grid, stretch)
        self.mesh = m
        self.dim, self.nx, self.ny, self.nz = dim, nx, ny, nz
        self.Q, self.QT = (9, 5) if dim == 2 else (19, 7)
        self.params = lbm_params(dim, nx, ny, nz, float(Ra), float(Pr), float(Ma), float(Thot), float(Tcold),
                                 m.dt, m.length_LB, STORE[storage], MODE[mode], int(device), 0)
        self.storage, self.mode = storage, mode
        h = ctypes.c_void_p()
        self._x = np.ascontiguousarray(m.x)
        self._y = np.ascontiguousarray(m.y)
        self._z = np.ascontiguousarray(m.z) if m.z is not None else None
        _chk(lib().lbm_create(ctypes.byref(self.params), _p(self._x), _p(self._y), _p(self._z), ctypes.byref(h)),
             "lbm_create")
        self.h = h
        if kernel != "auto":
            self.set_option(OPT_KERNEL, KERNELS[kernel])
        if nblocks:
            self.set_option(OPT_NBLOCKS, nblocks)

    def set_option(self, option: int, value: int):
        _chk(lib().lbm_set_option(self.h, int(option), int(value)), "lbm_set_option")

    def get_option(self, option: int) -> int:
        v = ctypes.c_int64()
        _chk(lib().lbm_get_option(self.h, int(option), ctypes.byref(v)), "lbm_get_option")
        return int(v.value)

    @property
    def kernel(self) -> str:
        return "march" if self.get_option(OPT_KERNEL) == 2 else "direct"

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().lbm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def shape(self):
        return (self.ny, self.nx) if self.dim == 2 else (self.nz, self.ny, self.nx)

    @property
    def nnode(self) -> int:
        return self.nx * self.ny * self.nz

    def derived(self) -> dict:
        out = np.zeros(9)
        _chk(lib().lbm_derived_params(ctypes.byref(self.params), _p(out)), "lbm_derived_params")
        keys = ["viscosity_LB", "kappa", "gbeta", "tauf", "Snu", "Sq", "sig_k", "dt", "length_LB"]
        return dict(zip(keys, out.tolist()))

    # initial(): 2M:136-281
    def initial(self):
        _chk(lib().lbm_init_reference(self.h), "lbm_init_reference")
        return self

    def init_equilibrium(self, rho, u, v, w, T):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, v, w, T)]
        _chk(lib().lbm_init_equilibrium(self.h, *[_p(a) for a in arrs]), "lbm_init_equilibrium")
        return self

    def init_warm(self, rho, u, v, w, T):
        """lbm_init_warm: equilibrium of the given fields plus the first-order
        non-equilibrium part from their gradients (warm starts)."""
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, v, w, T)]
        _chk(lib().lbm_init_warm(self.h, *[_p(a) for a in arrs]), "lbm_init_warm")
        return self

    def step(self, n: int = 1):
        _chk(lib().lbm_step(self.h, int(n)), "lbm_step")

    def run(self, max_steps: int, check_every: int = 2000, eps: float = float(np.float32(1e-6))):
        """lbm_run: iterate until both check() residuals are at most eps (tested
        every check_every iterations) or max_steps.  Returns (steps, errU, errT)."""
        n, a, b = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
        _chk(lib().lbm_run(self.h, int(max_steps), int(check_every), float(eps), ctypes.byref(n), ctypes.byref(a),
                           ctypes.byref(b)), "lbm_run")
        return int(n.value), a.value, b.value

    @property
    def itc(self) -> int:
        v = ctypes.c_int64()
        _chk(lib().lbm_itc(self.h, ctypes.byref(v)), "lbm_itc")
        return int(v.value)

    def check(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _chk(lib().lbm_check(self.h, ctypes.byref(a), ctypes.byref(b)), "lbm_check")
        return a.value, b.value

    def nusselt(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _chk(lib().lbm_nusselt(self.h, ctypes.byref(a), ctypes.byref(b)), "lbm_nusselt")
        return a.value, b.value

    def sums(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _chk(lib().lbm_sums(self.h, ctypes.byref(a), ctypes.byref(b)), "lbm_sums")
        return a.value, b.value

    def macro(self) -> dict:
        out = {k: np.zeros(self.shape) for k in ("rho", "u", "v", "w", "T")}
        _chk(lib().lbm_get_macro(self.h, *[_p(out[k]) for k in ("rho", "u", "v", "w", "T")]), "lbm_get_macro")
        if self.dim == 2:
            del out["w"]
        return out

    def get_macro_into(self, rho=None, u=None, v=None, w=None, T=None):
        """Copy the macroscopic fields into caller-owned float64 arrays (e.g. pinned)."""
        _chk(lib().lbm_get_macro(self.h, _p(rho), _p(u), _p(v), _p(w), _p(T)), "lbm_get_macro")

    def set_macro(self, rho=None, u=None, v=None, w=None, T=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, v, w, T)]
        _chk(lib().lbm_set_macro(self.h, *[_p(a) for a in arrs]), "lbm_set_macro")

    def populations(self):
        f = np.zeros(self.shape + (self.Q,))
        g = np.zeros(self.shape + (self.QT,))
        _chk(lib().lbm_get_populations(self.h, _p(f), _p(g)), "lbm_get_populations")
        return f, g

    def set_populations(self, f, g):
        f = np.ascontiguousarray(f, dtype=np.float64)
        g = np.ascontiguousarray(g, dtype=np.float64)
        assert f.size == self.nnode * self.Q and g.size == self.nnode * self.QT
        _chk(lib().lbm_set_populations(self.h, _p(f), _p(g)), "lbm_set_populations")

    def set_storage(self, storage: str):
        """lbm_set_storage: the state converted to another population storage
        in place, on the device (e.g. FP32 -> FP64 to finish a run)."""
        _chk(lib().lbm_set_storage(self.h, STORE[storage]), "lbm_set_storage")
        self.storage = storage

    def synchronize(self):
        _chk(lib().lbm_synchronize(self.h), "lbm_synchronize")

    def stream_ptr(self) -> int:
        s = ctypes.c_void_p()
        _chk(lib().lbm_stream(self.h, ctypes.byref(s)), "lbm_stream")
        return int(s.value or 0)

    def device_bytes(self) -> int:
        v = ctypes.c_int64()
        _chk(lib().lbm_device_bytes(self.h, ctypes.byref(v)), "lbm_device_bytes")
        return int(v.value)


# ---------------------------------------------------------------------------
# batches of cavities
# ---------------------------------------------------------------------------
class _Member(Cavity):
    """A member cavity of a Batch: an ordinary handle owned by the batch."""

    def __init__(self, batch, i, h, dim, nx, ny, nz, params, mesh_):
        self.h = h
        self.dim, self.nx, self.ny, self.nz = dim, nx, ny, nz
        self.Q, self.QT = (9, 5) if dim == 2 else (19, 7)
        self.params, self.mesh = params, mesh_
        self.storage, self.mode = batch.storage, batch.mode
        self._batch = batch

    def close(self):  # owned by the batch
        self.h = None


class Batch:
    """Many independent cavities advanced together (lbm_batch_*).  `specs` is
    a list of dicts with the Cavity keyword arguments (nx, ny, Ra, Pr, grid,
    stretch, coords, ...); dim, storage, mode and device are common to all
    members.  Without `coords` a member gets mesh_box with the physical aspect
    ny/nx (nz/nx), which is the reference's mesh for square members."""

    def __init__(self, dim, specs, storage="f64", mode="fast", device=0):
        self.dim, self.storage, self.mode = dim, storage, mode
        n = len(specs)
        P = (lbm_params * n)()
        self._keep = []
        xs, ys, zs = (_dp * n)(), (_dp * n)(), (_dp * n)()
        self._meshes = []
        for i, sp in enumerate(specs):
            nx, ny = int(sp["nx"]), int(sp["ny"])
            nz = int(sp.get("nz", 1)) if dim == 3 else 1
            # default: a box of physical size 1 x ny/nx (x nz/nx) -- the reference's
            # mesh() for square members, well-shaped cells for the others
            m = sp.get("coords") or mesh_box(nx, ny, nz if dim == 3 else 0, 1.0, ny / nx, nz / nx,
                                             sp.get("grid", "tanh"), sp.get("stretch", 1.5))
            self._meshes.append(m)
            P[i] = lbm_params(dim, nx, ny, nz, float(sp.get("Ra", 1e5)), float(sp.get("Pr", 0.71)),
                              float(sp.get("Ma", 0.1)), float(sp.get("Thot", 1.0)), float(sp.get("Tcold", 0.0)),
                              m.dt, m.length_LB, STORE[storage], MODE[mode], int(device), 0)
            arrs = [np.ascontiguousarray(a) for a in (m.x, m.y)] + ([np.ascontiguousarray(m.z)] if dim == 3 else [])
            self._keep += arrs
            xs[i], ys[i] = _p(arrs[0]), _p(arrs[1])
            if dim == 3:
                zs[i] = _p(arrs[2])
        self.specs = specs
        h = ctypes.c_void_p()
        _chk(lib().lbm_batch_create(n, P, xs, ys, zs if dim == 3 else None, ctypes.byref(h)), "lbm_batch_create")
        self.h = h
        self.n = n
        self.members = []
        for i in range(n):
            hh = ctypes.c_void_p()
            _chk(lib().lbm_batch_cavity(self.h, i, ctypes.byref(hh)), "lbm_batch_cavity")
            self.members.append(_Member(self, i, hh, dim, P[i].nx, P[i].ny, P[i].nz, P[i], self._meshes[i]))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().lbm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nodes(self):
        return sum(m.nnode for m in self.members)

    def initial(self):
        _chk(lib().lbm_batch_init_reference(self.h), "lbm_batch_init_reference")
        return self

    def step(self, n=1):
        _chk(lib().lbm_batch_step(self.h, int(n)), "lbm_batch_step")

    def synchronize(self):
        _chk(lib().lbm_batch_synchronize(self.h), "lbm_batch_synchronize")

    def check(self):
        a, b = np.zeros(self.n), np.zeros(self.n)
        _chk(lib().lbm_batch_check(self.h, _p(a), _p(b)), "lbm_batch_check")
        return a, b

    def nusselt(self):
        a, b = np.zeros(self.n), np.zeros(self.n)
        _chk(lib().lbm_batch_nusselt(self.h, _p(a), _p(b)), "lbm_batch_nusselt")
        return a, b

    def run(self, max_steps, check_every=2000, eps=float(np.float32(1e-6))):
        conv = (ctypes.c_int32 * self.n)()
        done = (ctypes.c_int64 * self.n)()
        _chk(lib().lbm_batch_run(self.h, int(max_steps), int(check_every), float(eps), conv, done), "lbm_batch_run")
        return np.array(conv[:], dtype=bool), np.array(done[:], dtype=np.int64)

    def run_masked(self, mask, max_steps, check_every=2000, eps=float(np.float32(1e-6))):
        """lbm_batch_run_masked: only members with mask[i] run.  Returns the
        status per member (1 converged, 0 not converged, -1 stopped for a
        diverging residual) and the steps each member did."""
        m = None if mask is None else (ctypes.c_int32 * self.n)(*[int(bool(v)) for v in mask])
        conv = (ctypes.c_int32 * self.n)()
        done = (ctypes.c_int64 * self.n)()
        _chk(lib().lbm_batch_run_masked(self.h, m, int(max_steps), int(check_every), float(eps), conv, done),
             "lbm_batch_run_masked")
        return np.array(conv[:], dtype=np.int32), np.array(done[:], dtype=np.int64)

    def run_mixed(self, mask, max_steps, check_every=2000, switch_eps=1e-5, eps=float(np.float32(1e-6))):
        """lbm_batch_run_mixed: FP32 to switch_eps, then each member on its own
        converted to FP64 and run to eps.  Returns (status, steps, FP32 steps)."""
        m = None if mask is None else (ctypes.c_int32 * self.n)(*[int(bool(v)) for v in mask])
        conv = (ctypes.c_int32 * self.n)()
        done = (ctypes.c_int64 * self.n)()
        low = (ctypes.c_int64 * self.n)()
        _chk(lib().lbm_batch_run_mixed(self.h, m, int(max_steps), int(check_every), float(switch_eps), float(eps),
                                       conv, done, low), "lbm_batch_run_mixed")
        self._sync_storage()
        return np.array(conv[:], dtype=np.int32), np.array(done[:], dtype=np.int64), np.array(low[:], np.int64)

    def tune(self, steps=20, storages=None):
        """lbm_batch_tune; storages: the storages the tuner may pick (names),
        None for the current one.  Returns the choice."""
        if storages is not None:
            self.set_option("storages", sum(1 << STORE[s] for s in storages))
        t, nb, v = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double()
        _chk(lib().lbm_batch_tune(self.h, int(steps), ctypes.byref(t), ctypes.byref(nb), ctypes.byref(v)),
             "lbm_batch_tune")
        self._sync_storage()
        return {"tile": t.value, "nblocks": nb.value, "mlups": v.value, "storage": self.storage}

    def set_storage(self, storage):
        """lbm_batch_set_storage: every member's state in another storage, in place."""
        _chk(lib().lbm_batch_set_storage(self.h, STORE[storage]), "lbm_batch_set_storage")
        self._sync_storage()

    def _sync_storage(self):
        code = self.get_option("storage")
        self.storage = {v: k for k, v in STORE.items()}.get(code, "mixed")
        for m in self.members:
            m.storage = self.storage

    def set_option(self, name, value):
        _chk(lib().lbm_batch_set_option(self.h, BATCH_OPT[name], int(value)), "lbm_batch_set_option")

    def get_option(self, name):
        v = ctypes.c_int64()
        _chk(lib().lbm_batch_get_option(self.h, BATCH_OPT[name], ctypes.byref(v)), "lbm_batch_get_option")
        return int(v.value)

    def stream_ptr(self):
        s = ctypes.c_void_p()
        _chk(lib().lbm_batch_stream(self.h, ctypes.byref(s)), "lbm_batch_stream")
        return int(s.value or 0)


def sweep_specs(n=256, seed=0, sides=(64, 96, 128, 192, 256, 384, 512), aspect=(1.0, 4.0),
                log10_ra=(3.0, 6.0), pr=(0.71, 7.0), stretch=(1.0, 2.0)):
    """The seeded parameter sweep of differentially heated 2D cavities: width
    from `sides`, height = width x aspect (tall cavities of physical size
    1 x aspect, mesh_box), Ra log-uniform, Pr and the tanh stretch uniform."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n):
        nx = int(rng.choice(sides))
        a = float(rng.uniform(*aspect))
        ny = int(round(nx * a))
        b = float(rng.uniform(*stretch))
        specs.append({"nx": nx, "ny": ny, "aspect": ny / nx, "Ra": float(10 ** rng.uniform(*log10_ra)),
                      "Pr": float(rng.uniform(*pr)), "grid": "tanh", "stretch": b,
                      "coords": mesh_box(nx, ny, 0, 1.0, ny / nx, 1.0, "tanh", b)})
    return specs


# ---------------------------------------------------------------------------
# program main (2M:283-380): loop with check every 2000 iterations
# ---------------------------------------------------------------------------
def run_main(cav: Cavity, itc_max: int = 20000, eps: float = float(np.float32(1e-6)),
             check_every: int = 2000, log=print):
    """The reference's driver loop: iterate while (errorU > epsU or errorT > epsT)
    and itc < itc_max, calling check() every `check_every` iterations and
    printing `itc errorU errorT` (2M:307-330, 800-802).  epsU = 1e-6 is a
    single-precision literal in the reference (2M:35), hence float32(1e-6).
    Returns (itc, errorU, errorT, seconds, MLUPS)."""
    errU = errT = 100.0
    itc = cav.itc
    t0 = time.perf_counter()
    while (errU > eps or errT > eps) and itc < itc_max:
        n = min(check_every - itc % check_every, itc_max - itc)
        cav.step(n)
        itc += n
        if itc % check_every == 0:
            errU, errT = cav.check()
            if log:
                log(f"{itc:12d}   {errU:.15E}   {errT:.15E}")
    cav.synchronize()
    dt = time.perf_counter() - t0
    mlups = cav.nnode / 1e6 * itc / dt if dt > 0 else float("nan")
    return itc, errU, errT, dt, mlups


def fortran_e(v: float, w: int, d: int) -> str:
    """Fortran `Ew.d` edit descriptor: 0.ddddE+xx right-justified in w columns."""
    v = float(v)
    if v == 0.0:
        s = "0." + "0" * d + "E+00"
    else:
        mant, ex = f"{abs(v):.{d - 1}E}".split("E")
        exp = int(ex) + 1
        s = "0." + mant.replace(".", "") + f"E{'+' if exp >= 0 else '-'}{abs(exp):02d}"
        if v < 0:
            s = "-" + s
    return s.rjust(w)


def write_tecplot(path: str, x, y, z, fields):
    """Tecplot POINT file in the reference's format, output_ASCII
    (2M:818-843: X Y U V T rho; 3M:1097-1121: X Y Z U V W RHO T), Fortran
    formats (1x,2(e11.4,' '),10(e13.6,' ')) and the ZONE line of format 101.
    x, y (, z): node coordinates c(0:n+1) with the walls; fields: arrays of
    shape (ny, nx) or (nz, ny, nx) (keys rho, u, v, [w,] T); z None in 2D."""
    e = fortran_e
    u = fields["u"]
    with open(path, "w") as fh:
        if z is None:
            ny, nx = u.shape
            fh.write(' TITLE="thermal convective flows"\n')
            fh.write(' VARIABLES="X" "Y" "U" "V" "T" "rho"\n')
            fh.write(f"ZONE I= {nx:5d}  J= {ny:5d} F=POINT\n")
            for j in range(ny):
                for i in range(nx):
                    vals = [fields["u"][j, i], fields["v"][j, i], fields["T"][j, i], fields["rho"][j, i]]
                    fh.write(" " + e(x[i + 1], 11, 4) + " " + e(y[j + 1], 11, 4) + " "
                             + " ".join(e(v, 13, 6) for v in vals) + " \n")
        else:
            nz, ny, nx = u.shape
            fh.write(' TITLE="side-heated convection "\n')
            fh.write(' VARIABLES="X" "Y" "Z" "U" "V" "W" "RHO" "T" \n')
            fh.write(f"ZONE I= {nx:5d}  J= {ny:5d} K= {nz:5d} F=POINT\n")
            for k in range(nz):
                for j in range(ny):
                    for i in range(nx):
                        vals = [z[k + 1], fields["u"][k, j, i], fields["v"][k, j, i], fields["w"][k, j, i],
                                fields["rho"][k, j, i], fields["T"][k, j, i]]
                        fh.write(" " + e(x[i + 1], 11, 4) + " " + e(y[j + 1], 11, 4) + " "
                                 + " ".join(e(v, 13, 6) for v in vals) + " \n")


def output_ascii(cav: Cavity, path: str):
    """The cavity's macroscopic fields (gathered from the GPU) as the
    reference's Tecplot file (write_tecplot)."""
    write_tecplot(path, cav.mesh.x, cav.mesh.y, cav.mesh.z if cav.dim == 3 else None, cav.macro())