"""The mbarrier protocol of the closure convolution (k_conv in
distributednavierstokes_b200/csrc/cnn.cuh), simulated on the host with
random interleavings of its roles:

* a producer loading input planes into a ring of nslot slots (full
  barriers, one TMA completion each; it refills a slot once its empty
  barrier's phase completes);
* two issuing lanes taking the sub-tiles in turn (sub-tile i on lane
  i % 2, accumulator i % 4, so each lane's accumulators are its own); both
  wait for every new plane of every tile, issue their sub-tiles' MMAs after
  the accumulator's release, commit tfull, and release each tile's
  last-used planes with a commit (empty barriers of two arrivals), then
  wait on their last tfull;
* four epilogue groups, group g taking sub-tiles i % 4 == g: wait tfull,
  read, release the accumulator (tempty, four arrivals).

A commit arrives once the committing lane's earlier MMAs are done; the
tensor pipe completes MMAs in issue order.  Checked: no deadlock; no parity
wait passes while its phase is incomplete, and none meets a barrier two
phases beyond it (which its parity test cannot tell from complete); no
slot is refilled while an MMA reading it is in flight; every MMA reads the
planes its tile needs.  The negative case shows why the kernel asserts one
epilogue group per accumulator: with three groups a group's wait can meet
its accumulator's barrier at the wrong phase.
"""
import random

import pytest


class Bar:
    def __init__(self, count):
        self.count, self.pend, self.done = count, 0, 0

    def arrive(self, k=1):
        self.pend += k
        assert self.pend <= self.count, "over-arrival"
        if self.pend == self.count:
            self.pend, self.done = 0, self.done + 1

    def test(self, parity, intended):
        """mbarrier.test_wait.parity: true when the phase of that parity is
        complete (the current phase's parity differs); `intended` is the
        phase index the caller means to wait for."""
        ok = (self.done & 1) != parity
        if ok:
            assert self.done >= intended + 1, ("spurious pass", self.done, intended)
        if self.done >= intended + 2:
            raise AssertionError(("aliased wait", self.done, intended))
        return ok


def simulate(ntiles, Do, z0, sub, nslot, seed, groups=4, nacc=4):
    rnd = random.Random(seed)
    tiles = []
    for t in range(z0, z0 + ntiles):
        z = t % Do
        tiles.append((t == z0 or z == 0, t == z0 + ntiles - 1 or z == Do - 1))
    full = [Bar(1) for _ in range(nslot)]
    empty = [Bar(2) for _ in range(nslot)]
    tfull = [Bar(1) for _ in range(nacc)]
    tempty = [Bar(4) for _ in range(nacc)]
    slot_plane = [None] * nslot
    mmas, commits, landing = [], [], []
    nsubs = ntiles * sub

    def producer():
        g = sl = ph = 0
        for fresh, _ in tiles:
            for _ in (range(3) if fresh else range(1)):
                while not empty[sl].test(ph ^ 1, g // nslot - 1):
                    yield
                assert not any(sl in m["slots"] and not m["done"] for m in mmas), "refill under an MMA"
                slot_plane[sl] = g
                landing.append(sl)
                g += 1
                sl += 1
                if sl == nslot:
                    sl, ph = 0, ph ^ 1
        yield "done"

    def lane(r):
        gs = gph = gid = 0
        sz, pg = [0, 0, 0], [0, 0, 0]
        i = 0
        last_a = last_i = -1
        for fresh, last in tiles:
            for _ in (range(3) if fresh else range(1)):
                while not full[gs].test(gph, gid // nslot):
                    yield
                sz, pg = [sz[1], sz[2], gs], [pg[1], pg[2], gid]
                gid += 1
                gs += 1
                if gs == nslot:
                    gs, gph = 0, gph ^ 1
            for sb in range(sub):
                ii = i + sb
                if ii % 2 != r:
                    continue
                ac, aph = ii % nacc, (ii // nacc) & 1
                while not tempty[ac].test(aph ^ 1, ii // nacc - 1):
                    yield
                assert all(slot_plane[sz[d]] == pg[d] for d in range(3))
                m = dict(lane=r, slots=set(sz), done=False)
                mmas.append(m)
                commits.append((r, len(mmas), tfull[ac]))
                last_a, last_i = ac, ii
                yield
            commits.append((r, len(mmas), empty[sz[0]]))
            if last:
                commits.append((r, len(mmas), empty[sz[1]]))
                commits.append((r, len(mmas), empty[sz[2]]))
            i += sub
            yield
        if last_a >= 0:
            while not tfull[last_a].test((last_i // nacc) & 1, last_i // nacc):
                yield
        yield "done"

    def epilogue(g):
        for ii in range(g, nsubs, groups):
            ac, aph = ii % nacc, (ii // nacc) & 1
            while not tfull[ac].test(aph, ii // nacc):
                yield
            yield
            tempty[ac].arrive(4)
        yield "done"

    def deliver():
        keep = []
        for ln, upto, bar in commits:
            if any(not m["done"] and m["lane"] == ln for m in mmas[:upto]):
                keep.append((ln, upto, bar))
            else:
                bar.arrive()
        commits[:] = keep

    actors = {"producer": producer(), "lane0": lane(0), "lane1": lane(1)}
    for g in range(groups):
        actors["group%d" % g] = epilogue(g)
    done, completed, steps = set(), 0, 0
    while len(done) < len(actors):
        steps += 1
        assert steps < 500_000, "no progress (deadlock)"
        c = rnd.random()
        if c < 0.15 and landing:
            full[landing.pop(0)].arrive()
        elif c < 0.35 and completed < len(mmas):
            mmas[completed]["done"] = True  # the pipe completes in issue order
            completed += 1
            deliver()
        elif c < 0.42 and commits:
            deliver()
        else:
            live = [k for k in actors if k not in done]
            k = rnd.choice(live)
            if next(actors[k]) == "done":
                done.add(k)


@pytest.mark.parametrize("sub", [1, 2, 3, 4])
@pytest.mark.parametrize("nslot", [4, 6])
def test_conv_protocol(sub, nslot):
    # (tiles of this CTA, tiles per column Do, first tile's position)
    for ntiles, Do, z0 in ((10, 5, 0), (7, 9, 2), (4, 1, 0), (8, 6, 3), (1, 4, 2)):
        for seed in range(6):
            simulate(ntiles, Do, z0, sub, nslot, seed)


def test_fewer_groups_than_accumulators_alias():
    failures = 0
    for seed in range(40):
        try:
            simulate(12, 6, 0, 3, 4, seed, groups=3)
        except AssertionError:
            failures += 1
    assert failures > 0
