"""CPU model of the TMA march kernels' schedule and shared-memory indexing.

The march kernels (csrc/lbm_march.cuh) fetch population boxes into ring
slots and compute every node from shared memory.  This model replays, for
many domain shapes and grid sizes, exactly the per-CTA schedule the kernels
run (segments, preloads, one prefetch per step, the slices each step waits
for) and every shared-memory element index the stencils touch, and checks:
  * each shared-memory index lies inside its box;
  * every slice a step reads was issued into its slot and not overwritten;
  * a slot is only refilled once no remaining step needs its slice;
  * no copy is left in flight at the end of a segment;
  * TMA box starts satisfy the 16-byte rule on the innermost coordinate;
  * the persistent CTAs cover every (tile, slice) work item exactly once.
"""
import itertools
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def off_a(i, n):
    return 1 if i == 0 else -1


def off_b(i, n):
    return 2 if i == 0 else (-2 if i == n - 1 else 1)


def need_lo(k, n):
    return k - 2 if k == n - 1 else (0 if k == 0 else k - 1)


def need_hi(k, n):
    return 2 if k == 0 else (k if k == n - 1 else k + 1)


def contiguous_plan(n, total, grid):
    """Per CTA, its segments (tile, first slice, end slice): an equal
    contiguous share of the (tile-major, slice-minor) items, split at tile
    boundaries (the 2D march kernel's own split)."""
    plan = []
    for b in range(grid):
        u, uend = total * b // grid, total * (b + 1) // grid
        segs = []
        while u < uend:
            t, ka = divmod(u, n)
            kb = ka + min(uend - u, n - ka)
            segs.append((t, ka, kb))
            u += kb - ka
        plan.append(segs)
    return plan


def library_plan(ntiles, nz, grid, kind):
    """The 3D march kernel's work plan as the library makes it (host code,
    no GPU needed)."""
    import ctypes
    from __graft_entry__ import load_package
    lib = load_package().lib()
    i32 = ctypes.c_int32
    fn = lib.lbm_march_plan3d
    fn.argtypes = [i32, i32, i32, i32, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i32),
                   ctypes.POINTER(i32)]
    cnt, used = i32(0), i32(0)
    assert fn(ntiles, nz, grid, kind, ctypes.byref(cnt), None, None, ctypes.byref(used)) == 0
    segs = (i32 * (3 * cnt.value))()
    off = (i32 * (used.value + 1))()
    assert fn(ntiles, nz, grid, kind, ctypes.byref(cnt), segs, off, ctypes.byref(used)) == 0
    return [[tuple(segs[3 * i:3 * i + 3]) for i in range(off[b], off[b + 1])] for b in range(used.value)]


def replay(n, total, plan, nodes_of_unit, check_node, ys=4, ns=2):
    """Replay the march schedule along an axis of n slices for the CTAs of
    `plan` (per CTA, its segments), with a ring of `ys` slots for the planes
    whose stencil reaches along the axis and `ns` slots for the others: at
    step k the copies of slices up to k + ys - 2 and k + ns - 1 are issued
    (the 3D kernel: 4 and 2; the 2D kernels: their layout's YS and NS).  The in-plane
    indices of a node do not depend on the step, so each tile's nodes are
    checked once, at every step kind (first, inner, last slice)."""
    covered = [0] * total
    checked = set()
    for segs in plan:
        slot = {}  # ring slot -> slice currently held
        nslot = {}
        inflight = set()
        for t, ka, kb in segs:
            assert 0 <= ka < kb <= n
            pre_lo, pre_hi = need_lo(ka, n), need_hi(ka, n)
            seg_hi = max(need_hi(kb - 1, n), pre_hi)

            def issue(s, k_now):
                assert 0 <= s < n
                old = slot.get(s % ys)
                if old is not None and old[0] == t:
                    # the slice being evicted must not be needed by this or a later step
                    for kk in range(k_now, kb):
                        assert not (need_lo(kk, n) <= old[1] <= need_hi(kk, n)), (old, kk)
                slot[s % ys] = (t, s)
                inflight.add(s)

            def issue_n(s, k_now):
                old = nslot.get(s % ns)
                assert old is None or old[0] != t or old[1] < k_now, (old, s, k_now)
                nslot[s % ns] = (t, s)

            y0 = min(seg_hi, max(pre_hi, ka + ys - 3))
            for s in range(pre_lo, y0 + 1):
                issue(s, ka)
            n0 = min(kb - 1, ka + ns - 2)
            for s in range(ka, n0 + 1):
                issue_n(s, ka)
            zissued, nissued = y0, n0
            for k in range(ka, kb):
                while zissued < min(seg_hi, k + ys - 2):
                    zissued += 1
                    issue(zissued, k)
                while nissued < min(kb - 1, k + ns - 1):
                    nissued += 1
                    issue_n(nissued, k)
                for s in range(need_lo(k, n), need_hi(k, n) + 1):
                    assert slot.get(s % ys) == (t, s), ("slice not resident", s, k)
                    inflight.discard(s)
                assert nslot[k % ns] == (t, k)
                kind = (t, 0 if k == 0 else (2 if k == n - 1 else 1))
                if kind not in checked:
                    checked.add(kind)
                    for node in nodes_of_unit(t):
                        check_node(node, k)
                covered[t * n + k] += 1
            assert not inflight, ("copies left in flight", inflight)
    assert all(c == 1 for c in covered)


# 3D: tiles of 32 x TY3 (x, y), TY3 = 8 or 4, boxes with +-HX columns and +-1 rows
TX3 = 32


def check_3d(nx, ny, nz, grid, es, TY3=8, kind=0):
    HX = 16 // es
    bx = lambda c: TX3 + (2 * HX if c & 1 else 0)  # noqa: E731
    by = lambda c: TY3 + (2 if c & 2 else 0)  # noqa: E731
    ntx, nty = -(-nx // TX3), -(-ny // TY3)
    ntiles = ntx * nty
    for tix in range(ntx):
        i0 = tix * TX3
        for c in range(4):
            x0 = i0 - (HX if c & 1 else 0)
            assert (x0 * es) % 16 == 0 and (bx(c) * es) % 16 == 0 and bx(c) <= 256 and by(c) <= 256

    def nodes(t):
        i0, j0 = (t % ntx) * TX3, (t // ntx) * TY3
        for ty, tx in itertools.product(range(TY3), range(TX3)):
            i, j = i0 + tx, j0 + ty
            if i < nx and j < ny:
                yield (tx, ty, i, j)

    def idx(c, tx, ty, dx, dy):
        r = ty + (1 if c & 2 else 0) + dy
        col = tx + (HX if c & 1 else 0) + dx
        assert 0 <= r < by(c) and 0 <= col < bx(c), (c, tx, ty, dx, dy)
        return r * bx(c) + col

    def check_node(node, k):
        tx, ty, i, j = node
        xa, xb, ya, yb = off_a(i, nx), off_b(i, nx), off_a(j, ny), off_b(j, ny)
        for c in range(4):
            idx(c, tx, ty, 0, 0)
        for dx in (xa, 0, xb):
            idx(1, tx, ty, dx, 0)
            for dy in (ya, 0, yb):
                idx(3, tx, ty, dx, dy)
        for dy in (ya, 0, yb):
            idx(2, tx, ty, 0, dy)
        for s in (k + off_a(k, nz), k, k + off_b(k, nz)):
            assert need_lo(k, nz) <= s <= need_hi(k, nz)

    replay(nz, ntiles * nz, library_plan(ntiles, nz, grid, kind), nodes, check_node)


def check_2d(nx, ny, grid, es, TX=128, ys=4, ns=2):
    HX = 16 // es
    bx = lambda c: TX + (2 * HX if c else 0)  # noqa: E731
    ntx = -(-nx // TX)
    for t in range(ntx):
        for c in range(2):
            x0 = t * TX - (HX if c else 0)
            assert (x0 * es) % 16 == 0 and (bx(c) * es) % 16 == 0 and bx(c) <= 256

    def nodes(t):
        for tx in range(TX):
            i = t * TX + tx
            if i < nx:
                yield (tx, i)

    def check_node(node, j):
        tx, i = node
        for c in range(2):
            for dx in (off_a(i, nx), 0, off_b(i, nx)):
                if c == 0 and dx:
                    continue
                col = tx + (HX if c else 0) + dx
                assert 0 <= col < bx(c)
        for s in (j + off_a(j, ny), j, j + off_b(j, ny)):
            assert need_lo(j, ny) <= s <= need_hi(j, ny)

    replay(ny, ntx * ny, contiguous_plan(ny, ntx * ny, grid), nodes, check_node, ys, ns)


@pytest.mark.parametrize("shape", [(128, 128, 128), (20, 16, 16), (33, 18, 7), (64, 24, 3), (40, 10, 5), (16, 16, 16),
                                   (96, 64, 40)])
@pytest.mark.parametrize("es", [8, 2])
@pytest.mark.parametrize("ty", [8, 4])
@pytest.mark.parametrize("kind", [0, 1])
def test_march3d_schedule_and_indices(shape, es, ty, kind):
    nx, ny, nz = shape
    if ny % ty == 1:
        pytest.skip("the host routes such shapes to the direct-load kernel")
    ntiles = -(-nx // TX3) * -(-ny // ty)
    total = ntiles * nz
    for grid in sorted({1, 3, 7, 128, 148, 256, 296, total}):
        if grid <= total:
            check_3d(nx, ny, nz, grid, es, ty, kind)


@pytest.mark.parametrize("ntiles,nz,grid", [(64, 128, 148), (128, 128, 296), (64, 128, 128), (16, 100, 148),
                                            (64, 256, 148)])
def test_march3d_plan_balances_the_sms(ntiles, nz, grid):
    # the balanced plan keeps every SM busy: the busiest block's work (slices
    # plus 1.5 slice times per segment start) is within 10 % of the even
    # share, and a grid that is a multiple of the tile count is pure lockstep
    plan = library_plan(ntiles, nz, grid, 0)
    assert len(plan) <= grid
    cost = [sum(kb - ka + 1.5 for _, ka, kb in segs) for segs in plan]
    ideal = ntiles * nz / grid + 1.5
    assert max(cost) <= 1.10 * ideal, (max(cost), ideal)
    if grid % ntiles == 0:
        assert len(plan) == grid and all(len(s) == 1 for s in plan)


@pytest.mark.parametrize("shape", [(2048, 64), (128, 128), (130, 9), (48, 48), (300, 3), (40, 24)])
@pytest.mark.parametrize("es", [8, 4, 2])
@pytest.mark.parametrize("tx", [32, 64, 128])
@pytest.mark.parametrize("ring", [(4, 2), (5, 3), (6, 4)])  # batch kernel 4 / 2, single-cavity kernel 6 / 4
def test_march2d_schedule_and_indices(shape, es, tx, ring):
    ys, ns = ring
    nx, ny = shape
    total = -(-nx // tx) * ny
    for grid in sorted({1, 2, 5, 148, 592, total}):
        if grid <= total:
            check_2d(nx, ny, grid, es, tx, ys, ns)
