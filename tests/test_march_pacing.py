"""CPU model of the march kernels' step pacing (csrc/lbm_march.cuh: march2d_run
over rows, march3d_run over z-slices; the same protocol).

The march kernels pace their steps with mbarriers instead of a block barrier
per step (described here for rows): one thread (in warp 0) issues the TMA copies of a y-ring of 4 slots
and a plane ring of 2 slots; before it overwrites the slots of rows j-2 / j-1
it waits for a "row done" barrier that every warp arrives on after each row
(two of them, by row parity); a block barrier starts each segment.  This model
runs that protocol for several warps under random interleavings and random
copy latencies, with the kernel's own ring bookkeeping (issue order, parity
bits, the slices each row waits for), and checks:
  * every slice a row reads has landed in its slot and was not overwritten;
  * each phase of a row-done barrier counts the arrivals of exactly one row;
  * the schedule never deadlocks and leaves no copy in flight at the end.
"""
import random

import pytest


def need_lo(k, n):
    return k - 2 if k == n - 1 else (0 if k == 0 else k - 1)


def need_hi(k, n):
    return 2 if k == 0 else (k if k == n - 1 else k + 1)


class Bar:
    """mbarrier: `count` arrivals (plus landed copies) complete a phase."""

    def __init__(self, count):
        self.count, self.pending, self.phase = count, 0, 0
        self.rows = []          # model only: the row each arrival of the current phase belongs to

    def test(self, parity):     # try_wait.parity: true once the phase of that parity completed
        return (self.phase & 1) != parity

    def arrive(self, row=None):
        self.pending += 1
        self.rows.append(row)
        if self.pending == self.count:
            if row is not None:
                assert len(set(self.rows)) == 1, f"one phase counted rows {self.rows}"
            self.phase += 1
            self.pending = 0
            self.rows = []


class Model:
    def __init__(self, nwarps, segments, rng):
        self.nw = nwarps
        self.segs = segments                    # [(ny, ja, jb)]
        self.rng = rng
        self.ybar = [Bar(1) for _ in range(4)]
        self.nbar = [Bar(1) for _ in range(2)]
        self.done = [Bar(nwarps) for _ in range(2)]
        self.yslot = [None] * 4                 # landed row per slot
        self.nslot = [None] * 2
        self.flight = []                        # (ring, slot, row)
        self.at_barrier = 0

    def land_one(self):
        k = self.rng.randrange(len(self.flight))
        ring, slot, row = self.flight.pop(k)
        if ring == "y":
            self.yslot[slot] = row
            self.ybar[slot].arrive()
        else:
            self.nslot[slot] = row
            self.nbar[slot].arrive()

    def warp(self, w):
        """The program of warp w, as in march2d_run; yields while it waits."""
        ynext = nnext = 0
        t = 0
        producer = w == 0

        def issue_y(s):
            nonlocal ynext
            if producer:
                assert (s & 3) not in [sl for r, sl, _ in self.flight if r == "y"], "slot refilled in flight"
                self.yslot[s & 3] = None
                self.flight.append(("y", s & 3, s))
            ynext ^= 1 << (s & 3)

        def issue_n(s):
            nonlocal nnext
            if producer:
                assert (s & 1) not in [sl for r, sl, _ in self.flight if r == "n"], "slot refilled in flight"
                self.nslot[s & 1] = None
                self.flight.append(("n", s & 1, s))
            nnext ^= 1 << (s & 1)

        for ny, ja, jb in self.segs:
            # segment-start block barrier
            self.at_barrier += 1
            gen = self.gen
            while not (self.gen != gen):
                if self.at_barrier == self.nw:
                    self.at_barrier = 0
                    self.gen += 1
                    break
                yield
            pre_lo, pre_hi = need_lo(ja, ny), need_hi(ja, ny)
            seg_hi = max(need_hi(jb - 1, ny), pre_hi)
            for s in range(pre_lo, pre_hi + 1):
                issue_y(s)
            issue_n(ja)
            yissued = pre_hi
            for j in range(ja, jb):
                iy = yissued < seg_hi and j + 2 <= seg_hi and j + 2 > yissued
                inn = j + 1 < jb
                if producer and (iy or inn) and j > ja:
                    while not self.done[(t - 1) & 1].test(((t - 1) >> 1) & 1):
                        yield
                if iy:
                    issue_y(j + 2)
                    yissued = j + 2
                if inn:
                    issue_n(j + 1)
                for s in range(need_lo(j, ny), need_hi(j, ny) + 1):
                    while not self.ybar[s & 3].test(((ynext >> (s & 3)) & 1) ^ 1):
                        yield
                while not self.nbar[j & 1].test(((nnext >> (j & 1)) & 1) ^ 1):
                    yield
                yield  # the row's arithmetic may interleave with others
                for s in range(need_lo(j, ny), need_hi(j, ny) + 1):
                    assert self.yslot[s & 3] == s, f"warp {w} row {j} read slot {s & 3} holding {self.yslot[s & 3]}"
                assert self.nslot[j & 1] == j, f"warp {w} row {j} plane slot holds {self.nslot[j & 1]}"
                yield
                self.done[t & 1].arrive(row=t)
                t += 1

    def run(self):
        self.gen = 0
        progs = [self.warp(w) for w in range(self.nw)]
        alive = list(range(self.nw))
        stall = 0
        while alive:
            if self.flight and self.rng.random() < 0.3:
                self.land_one()
                stall = 0
                continue
            w = self.rng.choice(alive)
            try:
                next(progs[w])
            except StopIteration:
                alive.remove(w)
            stall += 1
            assert stall < 20000 or self.flight, "deadlock: every warp waits and no copy is in flight"
            if stall >= 20000 and self.flight:
                self.land_one()
                stall = 0
        assert not self.flight, "copies left in flight"


SEGMENT_LISTS = [
    [(20, 0, 20)],                       # a whole column
    [(9, 0, 3), (9, 3, 9)],              # one column in two segments
    [(12, 4, 7)],                        # the middle
    [(10, 7, 10)],                       # the top wall
    [(6, 0, 1), (6, 1, 2), (6, 5, 6)],   # one-row segments, both walls
    [(5, 0, 5), (7, 2, 6), (3, 0, 3)],   # several cavities (a batch block)
    [(40, 0, 40), (8, 6, 8)],
]


@pytest.mark.parametrize("nwarps", [1, 2, 4])
@pytest.mark.parametrize("segs", SEGMENT_LISTS)
def test_row_pacing_is_race_free(nwarps, segs):
    for seed in range(40):
        Model(nwarps, segs, random.Random(seed * 7919 + nwarps)).run()
