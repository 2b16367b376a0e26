"""The N>1 host path on CPU: LPT sharding of independent cavities over ranks
and the final gather of per-cavity results, run as world_size-2 gloo process
groups (no GPU)."""
import os
import socket

import numpy as np
import pytest


def test_lpt_shards_cover_every_cavity_once(pkg):
    S = pkg.sharding
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 8):
        w = rng.integers(1, 500, size=37) ** 2
        sh = S.lpt_shards(w, world)
        assert len(sh) == world
        flat = sorted(i for s in sh for i in s)
        assert flat == list(range(37))
        loads = [sum(w[i] for i in s) for s in sh]
        # LPT bound: the spread between ranks is at most the largest item
        assert max(loads) - min(loads) <= max(w)


def test_lpt_is_deterministic_and_balanced_on_the_sweep(pkg):
    specs = pkg.sweep_specs(256, seed=0)
    a = pkg.sharding.lpt_shards([pkg.sharding.case_nodes(c) for c in specs], 8)
    b = pkg.sharding.lpt_shards([pkg.sharding.case_nodes(c) for c in specs], 8)
    assert a == b
    loads = [sum(pkg.sharding.case_nodes(specs[i]) for i in s) for s in a]
    assert max(loads) / min(loads) < 1.02


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    from __graft_entry__ import load_package
    pkg = load_package()
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cases = [{"nx": n, "ny": m} for n, m in zip(range(10, 40), range(50, 20, -1))]
        idx, mine = pkg.sharding.my_share(cases, world, rank)
        vals = {"nodes": [c["nx"] * c["ny"] for c in mine], "rank": [rank] * len(mine)}
        out = pkg.sharding.gather_by_index(idx, vals, len(cases))
        q.put((rank, idx, out["nodes"].tolist(), out["rank"].tolist()))
    finally:
        dist.destroy_process_group()


def test_gather_by_index_over_two_gloo_ranks(pkg):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    expect_nodes = [n * m for n, m in zip(range(10, 40), range(50, 20, -1))]
    idx0, idx1 = res[0][1], res[1][1]
    assert sorted(idx0 + idx1) == list(range(30)) and not set(idx0) & set(idx1)
    for rank, _, nodes, owner in res:
        assert nodes == expect_nodes            # every rank sees every cavity's result
        assert all(owner[i] == 0 for i in idx0) and all(owner[i] == 1 for i in idx1)
