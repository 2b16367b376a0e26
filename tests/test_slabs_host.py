"""The slab decomposition's host logic on CPU: the row partition and the
ghost-row exchange between ranks (slabs.exchange_ranks), run as gloo
process groups of 2 and 3 ranks with stand-in slabs that hold their rows in
host tensors (no GPU)."""
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


class FakeSlab:
    """Rows [y0, y1) of a (ny, 4) field plus ghost rows, in host tensors; the
    methods exchange_ranks calls, with the library's meaning of side 0 / 1."""

    def __init__(self, field, y0, y1):
        import torch
        self.torch = torch
        ny = field.shape[0]
        self.y0, self.y1 = y0, y1
        self.b0, self.b1 = (y0 - 1 if y0 > 0 else 0), (y1 + 1 if y1 < ny else ny)
        self.rows = torch.full((self.b1 - self.b0, field.shape[1]), float("nan"), dtype=torch.float64)
        self.rows[y0 - self.b0:y1 - self.b0] = torch.from_numpy(field[y0:y1])

    def halo_buffer(self):
        return self.torch.empty(self.rows.shape[1], dtype=self.torch.float64)

    def pack(self, side, buf):
        buf.copy_(self.rows[self.y0 - self.b0] if side == 0 else self.rows[self.y1 - 1 - self.b0])

    def unpack(self, side, buf):
        self.rows[0 if side == 0 else self.rows.shape[0] - 1] = buf

    def synchronize(self):
        pass


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import sys
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from __graft_entry__ import load_package
    pkg = load_package()
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ny = 11
        field = np.arange(ny * 4, dtype=np.float64).reshape(ny, 4)
        y0, y1 = pkg.slabs.partition_rows(ny, world)[rank]
        s = FakeSlab(field, y0, y1)
        pkg.slabs.exchange_ranks(s, rank, world)
        q.put((rank, s.b0, s.rows.numpy().copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ghost_rows_come_from_the_neighbouring_ranks(pkg, world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    field = np.arange(11 * 4, dtype=np.float64).reshape(11, 4)
    for rank, b0, rows in res:
        # after one exchange every row the slab holds, ghosts included, is the field's row
        assert np.array_equal(rows, field[b0:b0 + rows.shape[0]]), rank
