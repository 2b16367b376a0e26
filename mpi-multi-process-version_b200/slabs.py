"""One cavity split into slabs along its slowest axis: rows of y in 2D, z-slices
in 3D (lbm_create_slab, lbm_halo_*).

The reference decomposes its domain over MPI ranks in slabs (y in
natural-convection_2dim_mono.f90, z in 3dim_mono.f90; ghost layers of f_post /
g_post) and exchanges the ghost layers after every collision (`update`,
natural-convection_2dim_mono.f90:572-589, 2dim_block.f90:602-658,
3dim_mono.f90:732-749).  Here a slab is an ordinary handle over its layers plus
one ghost layer per neighbour; its step kernels compute only its own layers,
and after every step each interface swaps the boundary layers of all
population planes:

* `Slabs` keeps every slab in this process (one GPU, or one per listed device) and moves
  the layers with device copies;
* `RankSlab` is one slab per process of a torch.distributed group and moves the layers
  with point-to-point messages (NCCL between GPUs); the check and Nusselt sums are
  all-reduced.

A domain then needs to fit one GPU only when it is split; results are bit-identical
to the whole cavity's in exact mode (tested), the reductions equal to rounding.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import lbm as L


def partition_rows(n: int, nslabs: int) -> list[tuple[int, int]]:
    """Contiguous layer ranges [lo, hi) of near-equal size, at least 2 layers each."""
    if nslabs < 1 or n < 2 * nslabs:
        raise ValueError(f"{n} layers cannot make {nslabs} slabs of >= 2 layers")
    b = [n * s // nslabs for s in range(nslabs + 1)]
    return [(b[s], b[s + 1]) for s in range(nslabs)]


class Domain:
    """The whole domain a set of slabs shares: sizes, parameters, mesh.  nz = 0
    for a 2D domain (split along y), nz > 0 for a 3D one (split along z)."""

    def __init__(self, nx: int, ny: int, nz: int = 0, Ra: float = 1e5, Pr: float = 0.71, Ma: float = 0.1,
                 Thot: float = 1.0, Tcold: float = 0.0, grid: str = "erf", stretch: float = 3.2,
                 storage: str = "f64", mode: str = "fast", coords: L.Mesh | None = None):
        self.nx, self.ny, self.nz = nx, ny, int(nz)
        self.dim = 3 if self.nz else 2
        self.mesh = coords or L.mesh(nx, ny, self.nz, grid, stretch)
        self.args = (float(Ra), float(Pr), float(Ma), float(Thot), float(Tcold))
        self.storage, self.mode = storage, mode

    @property
    def nsplit(self) -> int:
        """Layers of the split axis (ny in 2D, nz in 3D)."""
        return self.ny if self.dim == 2 else self.nz

    @property
    def shape(self) -> tuple:
        return (self.ny, self.nx) if self.dim == 2 else (self.nz, self.ny, self.nx)

    def params(self, device: int) -> L.lbm_params:
        Ra, Pr, Ma, Th, Tc = self.args
        m = self.mesh
        return L.lbm_params(self.dim, self.nx, self.ny, max(self.nz, 1), Ra, Pr, Ma, Th, Tc, m.dt, m.length_LB,
                            L.STORE[self.storage], L.MODE[self.mode], int(device), 0)


class _Slab(L.Cavity):
    """A slab handle: an ordinary cavity over layers [b0, b1) of the whole
    domain's split axis (its own layers [y0, y1) plus ghost layers), created by
    lbm_create_slab.  y0, y1, b0, b1 count rows in 2D and z-slices in 3D."""

    def __init__(self, dom: Domain, y0: int, y1: int, device: int = 0, kernel: str = "auto"):
        p = dom.params(device)
        m = dom.mesh
        self._x, self._y = np.ascontiguousarray(m.x), np.ascontiguousarray(m.y)
        self._z = np.ascontiguousarray(m.z) if dom.dim == 3 else None
        h = ctypes.c_void_p()
        L._chk(L.lib().lbm_create_slab(ctypes.byref(p), L._p(self._x), L._p(self._y), L._p(self._z), int(y0),
                                       int(y1), ctypes.byref(h)), "lbm_create_slab")
        self.h = h
        self.y0, self.y1 = y0, y1
        self.b0 = y0 - 1 if y0 > 0 else 0
        self.b1 = y1 + 1 if y1 < dom.nsplit else dom.nsplit
        self.dim, self.nx = dom.dim, dom.nx
        if dom.dim == 2:
            self.ny, self.nz = self.b1 - self.b0, 1
            self.Q, self.QT = 9, 5
            self.mesh = L.Mesh(m.x, m.y[self.b0:self.b1 + 2], None, m.dx0, m.length_LB, m.dt)
        else:
            self.ny, self.nz = dom.ny, self.b1 - self.b0
            self.Q, self.QT = 19, 7
            self.mesh = L.Mesh(m.x, m.y, m.z[self.b0:self.b1 + 2], m.dx0, m.length_LB, m.dt)
        self.params, self.storage, self.mode = p, dom.storage, dom.mode
        self.device = device
        self.esize = 8 if dom.storage == "f64" else 4
        if kernel != "auto":
            self.set_option(L.OPT_KERNEL, L.KERNELS[kernel])

    @property
    def own(self) -> slice:
        """The slab's own layers within its fields (ghost layers left out)."""
        return slice(self.y0 - self.b0, self.y1 - self.b0)

    def halo_bytes(self) -> int:
        n = ctypes.c_int64(0)
        L._chk(L.lib().lbm_halo_size(self.h, ctypes.byref(n)), "lbm_halo_size")
        return int(n.value)

    def halo_buffer(self):
        import torch
        dt = torch.float64 if self.esize == 8 else torch.float32
        return torch.empty(self.halo_bytes() // self.esize, dtype=dt, device=f"cuda:{self.device}")

    def pack(self, side: int, buf):
        L._chk(L.lib().lbm_halo_pack(self.h, int(side), ctypes.c_void_p(buf.data_ptr())), "lbm_halo_pack")

    def unpack(self, side: int, buf):
        L._chk(L.lib().lbm_halo_unpack(self.h, int(side), ctypes.c_void_p(buf.data_ptr())), "lbm_halo_unpack")

    def check_sums(self) -> np.ndarray:
        s = np.zeros(4)
        L._chk(L.lib().lbm_check_sums(self.h, L._p(s)), "lbm_check_sums")
        return s

    def nusselt_sums(self) -> np.ndarray:
        s = np.zeros(3)
        L._chk(L.lib().lbm_nusselt_sums(self.h, L._p(s)), "lbm_nusselt_sums")
        return s


def _fields_of(fields, slab):
    """The layers of whole-domain fields ((ny, nx) or (nz, ny, nx)) a slab holds,
    ghost layers included."""
    return [None if a is None else np.ascontiguousarray(np.asarray(a, dtype=np.float64)[slab.b0:slab.b1])
            for a in fields]


class Slabs:
    """One cavity as `nslabs` slabs (rows in 2D, z-slices in 3D) in this
    process, on `devices` (one per slab, or all on one).  After every step each
    interface swaps its boundary layers (pack on both sides, wait, unpack): the
    ghost exchange of the reference's `update`.  check() and nusselt() combine
    the slabs' sums."""

    def __init__(self, dom: Domain, nslabs: int, devices=None, kernel: str = "auto"):
        self.dom = dom
        self.rows = partition_rows(dom.nsplit, nslabs)
        devs = list(devices) if devices is not None else [0] * nslabs
        if len(devs) == 1:
            devs = devs * nslabs
        self.slabs = [_Slab(dom, y0, y1, d, kernel) for (y0, y1), d in zip(self.rows, devs)]
        # buffers of each interface: the lower slab's top layer and the upper slab's bottom layer
        self._buf = [(lo.halo_buffer(), hi.halo_buffer()) for lo, hi in zip(self.slabs, self.slabs[1:])]

    def close(self):
        for s in self.slabs:
            s.close()
        self.slabs = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def initial(self):
        for s in self.slabs:
            s.initial()
        return self

    def init_equilibrium(self, rho, u, v, T, w=None):
        for s in self.slabs:
            r, a, b, t, c = _fields_of((rho, u, v, T, w), s)
            s.init_equilibrium(r, a, b, c, t)
        return self

    def exchange(self):
        """Swap every interface's boundary layers (the newest populations)."""
        for (lo, hi), (up_row, down_row) in zip(zip(self.slabs, self.slabs[1:]), self._buf):
            lo.pack(1, up_row)
            hi.pack(0, down_row)
        for s in self.slabs:
            s.synchronize()
        for (lo, hi), (up_row, down_row) in zip(zip(self.slabs, self.slabs[1:]), self._buf):
            if up_row.device != down_row.device:  # slabs on different GPUs: move the layers across
                import torch
                up_row, down_row = up_row.to(down_row.device), down_row.to(up_row.device)
                torch.cuda.synchronize(up_row.device)
                torch.cuda.synchronize(down_row.device)
            hi.unpack(0, up_row)
            lo.unpack(1, down_row)

    def step(self, n: int = 1):
        for _ in range(int(n)):
            for s in self.slabs:
                s.step(1)
            self.exchange()

    def synchronize(self):
        for s in self.slabs:
            s.synchronize()

    def macro(self) -> dict:
        """The whole domain's fields ((ny, nx) or (nz, ny, nx)), each slab's own layers."""
        keys = ("rho", "u", "v", "T") if self.dom.dim == 2 else ("rho", "u", "v", "w", "T")
        out = {k: np.zeros(self.dom.shape) for k in keys}
        for s in self.slabs:
            m = s.macro()
            for k in out:
                out[k][s.y0:s.y1] = m[k][s.own]
        return out

    def check(self):
        """errorU, errorT of the whole domain from the slabs' sums (2M:784, 798; 3M:1027-1082)."""
        t = sum(s.check_sums() for s in self.slabs)
        return float(np.sqrt(t[0]) / np.sqrt(t[1])), float(np.sqrt(t[2]) / np.sqrt(t[3]))

    def nusselt(self):
        t = sum(s.nusselt_sums() for s in self.slabs)
        return float(t[0] / t[2]), float(t[1] / t[2])


def exchange_ranks(slab, rank: int, world: int, group=None):
    """The ghost exchange of one slab per rank (torch.distributed): send the
    slab's boundary layers to the neighbouring ranks, receive theirs into its
    ghost layers.  `slab` needs halo_buffer(), pack(side, buf) and
    unpack(side, buf); rank r holds the r-th slab from the bottom."""
    import torch.distributed as dist
    ops, recv = [], []
    for side, peer in ((0, rank - 1), (1, rank + 1)):
        if 0 <= peer < world:
            out, inc = slab.halo_buffer(), slab.halo_buffer()
            slab.pack(side, out)
            slab.synchronize()
            ops.append(dist.P2POp(dist.isend, out, peer, group))
            ops.append(dist.P2POp(dist.irecv, inc, peer, group))
            recv.append((side, inc))
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()
        if recv and recv[0][1].is_cuda:  # the messages landed on torch's stream, the unpack runs on the slab's
            import torch
            torch.cuda.current_stream(recv[0][1].device).synchronize()
    for side, inc in recv:
        slab.unpack(side, inc)


class RankSlab(_Slab):
    """This rank's slab of a domain split over the ranks of a torch.distributed
    group (one slab per rank, NCCL between GPUs).  step() exchanges ghost layers
    after every iteration; check() and nusselt() all-reduce the sums."""

    def __init__(self, dom: Domain, rank: int, world: int, device: int = 0, kernel: str = "auto", group=None):
        y0, y1 = partition_rows(dom.nsplit, world)[rank]
        super().__init__(dom, y0, y1, device, kernel)
        self.rank, self.world, self.group = rank, world, group

    def step(self, n: int = 1):
        for _ in range(int(n)):
            super().step(1)
            exchange_ranks(self, self.rank, self.world, self.group)

    def _allreduce(self, v: np.ndarray) -> np.ndarray:
        import torch
        import torch.distributed as dist
        t = torch.tensor(v, dtype=torch.float64, device=f"cuda:{self.device}")
        dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()

    def check(self):
        t = self._allreduce(self.check_sums())
        return float(np.sqrt(t[0]) / np.sqrt(t[1])), float(np.sqrt(t[2]) / np.sqrt(t[3]))

    def nusselt(self):
        t = self._allreduce(self.nusselt_sums())
        return float(t[0] / t[2]), float(t[1] / t[2])
