"""A CPU model of the k_knn_tc pipeline's bookkeeping (sgt_knn.cu), checked
under random completion delays: the order in which the kernel issues bulk
copies, MMAs and tensor-memory scans, with the same stage, accumulator and
parity arithmetic.

- Tile ti lives in stage ti % nstage.  The wait for it is the mbarrier phase
  with parity (ti / nstage) & 1.
- Tile it goes to accumulator it & 1.  The wait for it is the phase with
  parity (it >> 1) & 1.
- The refill of a stage with tile pt + nstage follows the wait for MMA pt.
- Every iteration ends in a block barrier.

Invariants checked at every step:
- A wait on parity P succeeds only when the phase it means has completed,
  and its barrier is never a full phase ahead (no parity aliasing).
- A bulk copy never targets a stage that an unfinished MMA reads.
- An MMA never writes an accumulator whose previous tile is still being
  scanned.
- Every tile is multiplied exactly once and scanned exactly once, in order.
"""
import heapq

import numpy as np
import pytest


class Barrier:
    """mbarrier with arrival count 1: phases complete in order."""

    def __init__(self):
        self.completed = 0

    def try_wait(self, parity):
        # the phase with this parity has completed iff the current phase's
        # parity differs from it
        return (self.completed & 1) != parity


def run_model(nt, nstage, rng):
    t = 0.0
    events = []  # (time, seq, kind, payload)
    seq = [0]

    def schedule(delay, kind, payload):
        seq[0] += 1
        heapq.heappush(events, (t + delay, seq[0], kind, payload))

    barF = [Barrier() for _ in range(nstage)]
    barM = [Barrier(), Barrier()]
    stage_tile = [None] * nstage     # tile whose copy targets the stage
    stage_reader = [None] * nstage   # tile whose MMA reads the stage, until done
    acc_tile = [None, None]          # tile whose MMA writes the accumulator
    acc_scanning = [None, None]      # tile being scanned from the accumulator
    copies_issued, mma_done_tiles, scanned = [], [], []

    def advance_until(pred):
        nonlocal t
        while not pred():
            assert events, "deadlock: waited for an event that never comes"
            t, _, kind, payload = heapq.heappop(events)
            if kind == "copy":
                st, ti = payload
                assert stage_tile[st] == ti
                barF[st].completed += 1
                # the phase that completed is the one the tile's wait names
                assert barF[st].completed == ti // nstage + 1
            else:  # an MMA's commit
                s, ti = payload
                barM[s].completed += 1
                assert barM[s].completed == (ti >> 1) + 1
                st = ti % nstage
                assert stage_reader[st] == ti
                stage_reader[st] = None
                mma_done_tiles.append(ti)

    def load_tile(ti):
        st = ti % nstage
        # no MMA may still read the stage
        assert stage_reader[st] is None
        stage_tile[st] = ti
        copies_issued.append(ti)
        schedule(rng.exponential(3.0), "copy", (st, ti))

    for ti in range(min(nstage, nt)):
        load_tile(ti)
    for it in range(nt + 1):
        if it < nt:  # thread 0 issues the MMAs of tile it
            st, s = it % nstage, it & 1
            par = (it // nstage) & 1
            advance_until(lambda: barF[st].try_wait(par))
            # the wait really means tile it's copy, not a later or earlier one
            assert stage_tile[st] == it and barF[st].completed == it // nstage + 1
            # the accumulator's previous tile (it - 2) was scanned before the
            # last block barrier
            assert acc_scanning[s] is None
            acc_tile[s] = it
            stage_reader[st] = it
            schedule(rng.exponential(1.5), "mma", (s, it))
        if it >= 1:  # every warp scans tile it - 1
            pt, s = it - 1, (it - 1) & 1
            par = (pt >> 1) & 1
            advance_until(lambda: barM[s].try_wait(par))
            assert barM[s].completed == (pt >> 1) + 1
            assert acc_tile[s] == pt
            if pt + nstage < nt:
                load_tile(pt + nstage)
            acc_scanning[s] = pt
            t += rng.exponential(1.0)  # the scan itself
            scanned.append(pt)
            acc_scanning[s] = None  # block barrier: the scan is over
    return copies_issued, mma_done_tiles, scanned


@pytest.mark.parametrize("nstage", [2, 3])
@pytest.mark.parametrize("nt", [1, 2, 3, 7, 40])
def test_pipeline_bookkeeping(nt, nstage):
    rng = np.random.default_rng(nt * 10 + nstage)
    for _ in range(20):
        copies, mmas, scanned = run_model(nt, nstage, rng)
        assert copies == list(range(nt))
        assert sorted(mmas) == list(range(nt))
        assert scanned == list(range(nt))
