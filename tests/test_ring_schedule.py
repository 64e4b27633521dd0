"""A host model of the plane schedule of k_r4ring (csrc/r4.cuh), checked on
the CPU under random interleavings of the CTA's plane groups.

The kernel's rules, restated:
- CTA b walks the units u = b, b + G, ... (IL planes each); local plane k
  belongs to group k % NG (NG = IL) and lives in buffer k % NB (NB = NG + 1);
- the first NB planes are issued at the start; plane k + NB is issued into
  buffer k % NB once the group that used it for plane k is done with it --
  right after its last exchange (per-thread stores), or, with a store that
  reads the buffer (TMA tensor / bulk copy), at the group's next plane or
  after its last one;
- a group waits for use n = k // NB of its buffer by first waiting until the
  buffer's issue counter exceeds n, then on the mbarrier phase parity n & 1.

The model checks that every plane is processed exactly once, that no buffer
is refilled while its plane is still in use, that the parity wait always
sees the right phase, and that no interleaving deadlocks.  It also shows
why the issue counter is needed: with a parity wait alone some interleaving
accepts a phase two behind.
"""
import random

import pytest


def _run(G, IL, seed, deferred, guard=True):
    NG, NB = IL, IL + 1
    nunits = 4096 // IL
    seen = [0] * 4096
    rnd = random.Random(seed)
    for b in range(G):
        nloc = ((nunits - 1 - b) // G + 1) * IL if b < nunits else 0
        plane_of = lambda k: (b + (k // IL) * G) * IL + k % IL
        completed, content = [0] * NB, [None] * NB
        inflight, issued = [None] * NB, [0] * NB
        for k in range(min(NB, nloc)):
            inflight[k] = k
            issued[k] = 1
        nxt = {g: g for g in range(NG)}
        busy, pend, done = {}, {g: None for g in range(NG)}, set()

        def refill(kk):
            bf = kk % NB
            assert content[bf] is None and inflight[bf] is None
            if kk + NB < nloc:
                inflight[bf] = kk + NB
                issued[bf] += 1

        for _ in range(10 ** 6):
            for bf in range(NB):                       # copies land at random moments
                if inflight[bf] is not None and rnd.random() < 0.5:
                    content[bf], inflight[bf] = inflight[bf], None
                    completed[bf] += 1
            active = [g for g in range(NG) if g not in done]
            if not active:
                break
            g = rnd.choice(active)
            if g in busy:                              # the group finishes its plane
                k = busy.pop(g)
                content[k % NB] = None
                nxt[g] = k + NG
                if deferred:
                    pend[g] = k
                    if nxt[g] >= nloc:
                        refill(pend[g])
                        pend[g] = None
                        done.add(g)
                else:
                    refill(k)
                    if nxt[g] >= nloc:
                        done.add(g)
            else:                                      # the group waits for its next plane
                k = nxt[g]
                if k >= nloc:
                    done.add(g)
                    continue
                bf, n = k % NB, k // NB
                ready = (not guard or issued[bf] > n) and (completed[bf] & 1) != (n & 1)
                if ready:
                    if completed[bf] != n + 1 or content[bf] != k:
                        return False                   # a phase from another use was accepted
                    seen[plane_of(k)] += 1
                    busy[g] = k
                    if deferred and pend[g] is not None:
                        refill(pend[g])
                        pend[g] = None
        else:
            raise AssertionError("deadlock")
        assert all(x is None for x in inflight)
    assert all(x == 1 for x in seen)
    return True


@pytest.mark.parametrize("deferred", [False, True])
@pytest.mark.parametrize("IL", [2, 4])
@pytest.mark.parametrize("G", [148, 132, 7, 1])
def test_ring_schedule(G, IL, deferred):
    for seed in range(3):
        assert _run(G, IL, seed, deferred)


def test_parity_wait_alone_can_alias():
    """Without the issue counter a group can accept phase n - 2 of a buffer."""
    assert not all(_run(148, 2, seed, False, guard=False) for seed in range(20))
