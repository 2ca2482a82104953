"""The barrier protocol of the tensor-core chain's lane-major epilogue
(blade_b200/csrc/beamform_tc.cu, epilogue_transposed), as a model: two MMA
issuers, two Re warps and two Im warps over two accumulators, run in random
interleavings.  An mbarrier wait tests only the parity of the phase it waits
for, so a barrier that completes two phases before a waiter looks leaves that
waiter blocked (or, one phase later, passed at the wrong time).  The model checks
that every wait passes on exactly the phase it means and that no schedule
deadlocks; it also keeps the form that failed (the Re warps' handoff of the
range's last tile with nothing to gate it) to show that the check sees the
fault.  CPU only."""

import random

import pytest


class Bar:
    def __init__(self, count):
        self.count, self.pending, self.done = count, 0, 0

    def arrive(self):
        self.pending += 1
        if self.pending == self.count:
            self.pending, self.done = 0, self.done + 1


def run(n, nacc, nis, gated, seed):
    rnd = random.Random(seed)
    d_full = [Bar(1) for _ in range(nacc)]
    d_empty = [Bar(4) for _ in range(nacc)]  # two Re and two Im warps
    pr_full = [Bar(2) for _ in range(nacc)]  # the two Re warps
    faults = []

    def wait(bar, phase):
        while True:
            if bar.done % 2 != phase % 2:  # try_wait.parity: the phase of this parity is complete
                if bar.done != phase + 1:
                    faults.append(("wrong phase", phase, bar.done))
                return
            yield "blocked"

    def issuer(j):
        for k in range(j, n, nis):
            if k >= nacc:
                yield from wait(d_empty[k % nacc], k // nacc - 1)
            yield "mma"
            d_full[k % nacc].arrive()

    def re_warp():
        for k in range(n):
            yield from wait(d_full[k % nacc], k // nacc)
            yield "tmem"
            d_empty[k % nacc].arrive()
            if k:
                pr_full[(k - 1) % nacc].arrive()  # the previous tile's partial sums
            yield "store"
        # the last tile: first wait until tile n - nacc's accumulator is released
        # (the Im warps release it only after their wait for tile n - 1 - nacc)
        if gated and n >= nacc:
            yield from wait(d_empty[(n - nacc) % nacc], (n - nacc) // nacc)
        pr_full[(n - 1) % nacc].arrive()

    def im_warp():
        for k in range(n):
            yield from wait(d_full[k % nacc], k // nacc)
            yield "tmem"
            if k:
                yield from wait(pr_full[(k - 1) % nacc], (k - 1) // nacc)
            d_empty[k % nacc].arrive()
            yield "combine"
        yield from wait(pr_full[(n - 1) % nacc], (n - 1) // nacc)

    actors = [issuer(j) for j in range(nis)] + [re_warp(), re_warp(), im_warp(), im_warp()]
    alive = list(range(len(actors)))
    idle = 0
    while alive:
        i = rnd.choice(alive)
        try:
            step = next(actors[i])
        except StopIteration:
            alive.remove(i)
            idle = 0
            continue
        idle = idle + 1 if step == "blocked" else 0
        if idle > 200 * len(alive):
            return ["deadlock"] + faults
        if faults:
            return faults
    return faults


@pytest.mark.parametrize("nacc,nis", [(2, 1), (2, 2), (1, 1), (4, 2)])
def test_lane_major_epilogue_protocol_has_no_phase_aliasing(nacc, nis):
    for seed in range(1500):
        n = 1 + seed % 11
        assert run(n, nacc, nis, True, seed) == [], (n, seed)


def test_model_catches_the_ungated_last_handoff():
    bad = sum(1 for seed in range(1500) if run(1 + seed % 9, 2, 2, False, seed))
    assert bad > 0
