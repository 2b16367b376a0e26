"""One 2D cavity split into row slabs (lbm_create_slab, lbm_halo_*).

The reference decomposes its domain over MPI ranks (natural-convection_2dim_block.f90:
StartEnd, ghost rows of f_post / g_post) and exchanges the ghost rows after every
collision (`update`, natural-convection_2dim_mono.f90:572-589, 2dim_block.f90:602-658).
Here a slab is an ordinary handle over its rows plus one ghost row per neighbour; its
step kernels compute only its own rows, and after every step each interface swaps the
boundary rows of all population planes:

* `Slabs` keeps every slab in this process (one GPU, or one per listed device) and moves
  the rows with device copies;
* `RankSlab` is one slab per process of a torch.distributed group and moves the rows with
  point-to-point messages (NCCL between GPUs); the check and Nusselt sums are all-reduced.

Both need a domain that fits one GPU only when it is split; results are bit-identical to
the whole cavity's in exact mode (tested), the reductions equal to rounding.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import lbm as L


def partition_rows(ny: int, nslabs: int) -> list[tuple[int, int]]:
    """Contiguous row ranges [y0, y1) of near-equal size, at least 2 rows each."""
    if nslabs < 1 or ny < 2 * nslabs:
        raise ValueError(f"{ny} rows cannot make {nslabs} slabs of >= 2 rows")
    b = [ny * s // nslabs for s in range(nslabs + 1)]
    return [(b[s], b[s + 1]) for s in range(nslabs)]


class Domain:
    """The whole 2D domain a set of slabs shares: sizes, parameters, mesh."""

    def __init__(self, nx: int, ny: int, Ra: float = 1e5, Pr: float = 0.71, Ma: float = 0.1, Thot: float = 1.0,
                 Tcold: float = 0.0, grid: str = "erf", stretch: float = 3.2, storage: str = "f64",
                 mode: str = "fast", coords: L.Mesh | None = None):
        self.nx, self.ny = nx, ny
        self.mesh = coords or L.mesh(nx, ny, 0, grid, stretch)
        self.args = (float(Ra), float(Pr), float(Ma), float(Thot), float(Tcold))
        self.storage, self.mode = storage, mode

    def params(self, device: int) -> L.lbm_params:
        Ra, Pr, Ma, Th, Tc = self.args
        m = self.mesh
        return L.lbm_params(2, self.nx, self.ny, 1, Ra, Pr, Ma, Th, Tc, m.dt, m.length_LB, L.STORE[self.storage],
                            L.MODE[self.mode], int(device), 0)


class _Slab(L.Cavity):
    """A slab handle: an ordinary cavity over rows [b0, b1) of the whole domain
    (its own rows [y0, y1) plus ghost rows), created by lbm_create_slab."""

    def __init__(self, dom: Domain, y0: int, y1: int, device: int = 0, kernel: str = "auto"):
        p = dom.params(device)
        m = dom.mesh
        self._x, self._y = np.ascontiguousarray(m.x), np.ascontiguousarray(m.y)
        h = ctypes.c_void_p()
        L._chk(L.lib().lbm_create_slab(ctypes.byref(p), L._p(self._x), L._p(self._y), int(y0), int(y1),
                                       ctypes.byref(h)), "lbm_create_slab")
        self.h = h
        self.y0, self.y1 = y0, y1
        self.b0 = y0 - 1 if y0 > 0 else 0
        self.b1 = y1 + 1 if y1 < dom.ny else dom.ny
        self.dim, self.nx, self.ny, self.nz = 2, dom.nx, self.b1 - self.b0, 1
        self.Q, self.QT = 9, 5
        self.params, self.storage, self.mode = p, dom.storage, dom.mode
        self.mesh = L.Mesh(m.x, m.y[self.b0:self.b1 + 2], None, m.dx0, m.length_LB, m.dt)
        self.device = device
        self.esize = 8 if dom.storage == "f64" else 4
        if kernel != "auto":
            self.set_option(L.OPT_KERNEL, L.KERNELS[kernel])

    @property
    def own(self) -> slice:
        """The slab's own rows within its fields (ghost rows left out)."""
        return slice(self.y0 - self.b0, self.y1 - self.b0)

    def halo_buffer(self):
        import torch
        dt = torch.float64 if self.esize == 8 else torch.float32
        return torch.empty((self.Q + self.QT) * self.nx, dtype=dt, device=f"cuda:{self.device}")

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
    """The rows of whole-domain fields (ny, nx) a slab holds, ghost rows included."""
    return [None if a is None else np.ascontiguousarray(np.asarray(a, dtype=np.float64)[slab.b0:slab.b1])
            for a in fields]


class Slabs:
    """One 2D cavity as `nslabs` row slabs in this process, on `devices` (one
    per slab, or all on one).  After every step each interface swaps its
    boundary rows (pack on both sides, wait, unpack): the ghost exchange of
    the reference's `update`.  check() and nusselt() combine the slabs' sums."""

    def __init__(self, dom: Domain, nslabs: int, devices=None, kernel: str = "auto"):
        self.dom = dom
        self.rows = partition_rows(dom.ny, nslabs)
        devs = list(devices) if devices is not None else [0] * nslabs
        if len(devs) == 1:
            devs = devs * nslabs
        self.slabs = [_Slab(dom, y0, y1, d, kernel) for (y0, y1), d in zip(self.rows, devs)]
        # buffers of each interface: the lower slab's top row and the upper slab's bottom row
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

    def init_equilibrium(self, rho, u, v, T):
        for s in self.slabs:
            r, a, b, t = _fields_of((rho, u, v, T), s)
            s.init_equilibrium(r, a, b, None, t)
        return self

    def exchange(self):
        """Swap every interface's boundary rows (the newest populations)."""
        for (lo, hi), (up_row, down_row) in zip(zip(self.slabs, self.slabs[1:]), self._buf):
            lo.pack(1, up_row)
            hi.pack(0, down_row)
        for s in self.slabs:
            s.synchronize()
        for (lo, hi), (up_row, down_row) in zip(zip(self.slabs, self.slabs[1:]), self._buf):
            if up_row.device != down_row.device:  # slabs on different GPUs: move the rows across
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
        """The whole domain's fields (ny, nx), each slab's own rows."""
        out = {k: np.zeros((self.dom.ny, self.dom.nx)) for k in ("rho", "u", "v", "T")}
        for s in self.slabs:
            m = s.macro()
            for k in out:
                out[k][s.y0:s.y1] = m[k][s.own]
        return out

    def check(self):
        """errorU, errorT of the whole domain from the slabs' sums (2M:784, 798)."""
        t = sum(s.check_sums() for s in self.slabs)
        return float(np.sqrt(t[0]) / np.sqrt(t[1])), float(np.sqrt(t[2]) / np.sqrt(t[3]))

    def nusselt(self):
        t = sum(s.nusselt_sums() for s in self.slabs)
        return float(t[0] / t[2]), float(t[1] / t[2])


def exchange_ranks(slab, rank: int, world: int, group=None):
    """The ghost exchange of one slab per rank (torch.distributed): send the
    slab's boundary rows to the neighbouring ranks, receive theirs into its
    ghost rows.  `slab` needs halo_buffer(), pack(side, buf) and
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
    group (one slab per rank, NCCL between GPUs).  step() exchanges ghost rows
    after every iteration; check() and nusselt() all-reduce the sums."""

    def __init__(self, dom: Domain, rank: int, world: int, device: int = 0, kernel: str = "auto", group=None):
        y0, y1 = partition_rows(dom.ny, world)[rank]
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
