"""The slab decomposition's host logic on CPU: the layer partition, the
argument checks of lbm_create_slab, and the ghost exchange between ranks
(slabs.exchange_ranks), run as gloo process groups of 2 and 3 ranks with
stand-in slabs that hold their layers (rows of a 2D field, z-slices of a 3D
one) in host tensors (no GPU)."""
import ctypes
import os
import socket

import numpy as np
import pytest


def test_partition_rows_covers_the_domain(pkg):
    P = pkg.slabs.partition_rows
    for ny in (4, 7, 100, 2048):
        for n in range(1, min(ny // 2, 9) + 1):
            rows = P(ny, n)
            assert rows[0][0] == 0 and rows[-1][1] == ny
            assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
            assert all(y1 - y0 >= 2 for y0, y1 in rows)
            assert max(y1 - y0 for y0, y1 in rows) - min(y1 - y0 for y0, y1 in rows) <= 1
    with pytest.raises(ValueError):
        P(5, 3)


def test_create_slab_checks_its_arguments(pkg):
    """Argument errors come back before any device work (so also without a GPU)."""
    L = pkg.lbm
    for dim, n in ((2, (16, 12, 0)), (3, (16, 12, 10))):
        m = L.mesh(*n)
        dom = pkg.slabs.Domain(*n, coords=m)
        p = dom.params(0)
        z = L._p(m.z) if dim == 3 else None
        h = ctypes.c_void_p()
        nsplit = n[1] if dim == 2 else n[2]
        for lo, hi in ((-1, 4), (0, 1), (5, 6), (nsplit - 3, nsplit + 1)):
            st = L.lib().lbm_create_slab(ctypes.byref(p), L._p(m.x), L._p(m.y), z, lo, hi, ctypes.byref(h))
            assert st == -1, (dim, lo, hi)
            assert b"slab layers" in L.lib().lbm_last_error()
    # 3D without z coordinates
    m = L.mesh(16, 12, 10)
    p = pkg.slabs.Domain(16, 12, 10, coords=m).params(0)
    assert L.lib().lbm_create_slab(ctypes.byref(p), L._p(m.x), L._p(m.y), None, 0, 5, ctypes.byref(h)) == -1
    assert b"coordinates" in L.lib().lbm_last_error()


def test_domain_splits_the_slowest_axis(pkg):
    d2 = pkg.slabs.Domain(16, 12, coords=pkg.lbm.mesh(16, 12, 0))
    d3 = pkg.slabs.Domain(16, 12, 10, coords=pkg.lbm.mesh(16, 12, 10))
    assert (d2.dim, d2.nsplit, d2.shape) == (2, 12, (12, 16))
    assert (d3.dim, d3.nsplit, d3.shape) == (3, 10, (10, 12, 16))
    assert d3.params(0).nz == 10 and d2.params(0).nz == 1


class FakeSlab:
    """Layers [y0, y1) of a field (rows of an (ny, 4) field, or z-slices of an
    (nz, 3, 4) one) plus ghost layers, in host tensors; the methods
    exchange_ranks calls, with the library's meaning of side 0 / 1."""

    def __init__(self, field, y0, y1):
        import torch
        self.torch = torch
        ny = field.shape[0]
        self.y0, self.y1 = y0, y1
        self.b0, self.b1 = (y0 - 1 if y0 > 0 else 0), (y1 + 1 if y1 < ny else ny)
        self.rows = torch.full((self.b1 - self.b0,) + field.shape[1:], float("nan"), dtype=torch.float64)
        self.rows[y0 - self.b0:y1 - self.b0] = torch.from_numpy(field[y0:y1])

    def halo_buffer(self):
        return self.torch.empty(self.rows[0].numel(), dtype=self.torch.float64)

    def pack(self, side, buf):
        buf.copy_((self.rows[self.y0 - self.b0] if side == 0 else self.rows[self.y1 - 1 - self.b0]).reshape(-1))

    def unpack(self, side, buf):
        self.rows[0 if side == 0 else self.rows.shape[0] - 1] = buf.reshape(self.rows.shape[1:])

    def synchronize(self):
        pass


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _field(layered):
    return (np.arange(11 * 12, dtype=np.float64).reshape(11, 3, 4) if layered
            else np.arange(11 * 4, dtype=np.float64).reshape(11, 4))


def _worker(rank, world, port, q, layered=False):
    import datetime
    import sys
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from __graft_entry__ import load_package
    pkg = load_package()
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        field = _field(layered)
        y0, y1 = pkg.slabs.partition_rows(field.shape[0], world)[rank]
        s = FakeSlab(field, y0, y1)
        pkg.slabs.exchange_ranks(s, rank, world)
        q.put((rank, s.b0, s.rows.numpy().copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("layered", [False, True], ids=["rows", "zslices"])
@pytest.mark.parametrize("world", [2, 3])
def test_ghost_rows_come_from_the_neighbouring_ranks(pkg, world, layered):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, layered)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    field = _field(layered)
    for rank, b0, rows in res:
        # after one exchange every layer the slab holds, ghosts included, is the field's layer
        assert np.array_equal(rows, field[b0:b0 + rows.shape[0]]), rank
