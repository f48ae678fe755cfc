"""Host logic of the particle-mesh cutoff autotuner (bd_b200.autotune_pme_cutoff)
on CPU, with stand-in contexts: candidates past 0.43 L are skipped, every
other candidate is timed from its device-event slot after one untimed call,
each context is closed, the fastest wins, and a box that fits none is an
error.  (The GPU test in tests/test_gpu_pme.py runs it on real contexts.)"""
import numpy as np
import pytest

import bd_b200 as B


class FakeContext:
    """Answers the calls the autotuner makes; a product 'costs' ms(rc)."""

    def __init__(self, rc, ms, log):
        self.rc, self.ms, self.log = rc, ms, log
        self.N = 10
        self.calls = 0
        self.profiling = False
        self.total = 0.0
        self.count = 0
        self.closed = False

    def mobility_apply_block(self, V):
        assert V.shape == (4, 3 * self.N)
        self.calls += 1
        if self.profiling:
            self.total += self.ms
            self.count += 1
        return np.zeros_like(V)

    def profile(self, on=True):
        self.profiling = bool(on)
        if on:
            self.total, self.count = 0.0, 0

    def profile_read(self, slot):
        assert slot == B.Context.PROF_BLOCK
        return self.total, self.count

    def close(self):
        self.closed = True
        self.log.append(self)


def test_picks_the_fastest_fitting_candidate_and_closes_every_context():
    cost = {10.0: 2.0, 12.1: 1.5, 13.6: 1.2, 15.5: 1.4, 20.0: 0.1}
    closed = []
    best, times = B.autotune_pme_cutoff(lambda rc: FakeContext(rc, cost[rc], closed), 40.0, 4,
                                        candidates=tuple(cost), reps=3)
    # 20 > 0.43 * 40 = 17.2: never built
    assert sorted(times) == [10.0, 12.1, 13.6, 15.5]
    assert best == 13.6
    assert times == pytest.approx({rc: cost[rc] for rc in times})
    assert len(closed) == 4 and all(c.closed and c.calls == 4 for c in closed)


def test_box_too_small_for_every_candidate():
    with pytest.raises(ValueError):
        B.autotune_pme_cutoff(lambda rc: FakeContext(rc, 1.0, []), 20.0, 4,
                              candidates=(10.0, 12.1))
