"""Exhaustive check of the stage hand-off protocol of the SpMV pipelines
(k_spmv_pipe and k_spmv_xs in cfdrs_b200/csrc/kernels.cuh): one producer and
W consumer warps on a ring of S stages, each stage with a `full` and an
`empty` mbarrier. Every interleaving of the model is explored (breadth first).

Model of an mbarrier: K = number of completed phases; a parity wait on P
succeeds when (K & 1) != P (the phase of parity P has completed, as
mbarrier.try_wait.parity reports it). `full[s]` completes a phase when the
producer has filled stage s; `empty[s]` when all W warps have arrived.

Producer, block `it`: stage s = it % S; from it >= S it waits on empty[s]
with parity ((it / S) - 1) & 1, then fills the stage with block `it`.
Consumer warp, block `it`: waits on full[s] with parity (it / S) & 1 by
itself (no CTA barrier), reads the stage (a separate step, so the producer
may run in between), then arrives on empty[s].

Checked: every read sees the block the warp expects (the producer never
refills a stage a warp still reads, and no warp passes a wait for a phase
other than the one it means), every warp takes every block, nothing
deadlocks. A wrong parity formula must be caught (negative control)."""
from collections import deque

import pytest


def explore(W, S, B, consumer_parity=lambda it, S: (it // S) & 1, producer_waits=True,
            long_block=lambda it: False, reset_before_arrive=True):
    """Returns (states visited, first violation or None). Blocks for which
    long_block(it) holds take the long-row path: after reading, every warp
    posts its partial to the stage's counter (tagged with its block); warp 0
    waits for W posts, checks they all belong to its block, resets the
    counter and only then arrives (reset_before_arrive=False resets after)."""
    # state: producer block, per-warp (block, step), full K, empty K, empty pending,
    #        stage contents, per-stage posted partials (block tags)
    start = (0, tuple((0, 0) for _ in range(W)), (0,) * S, (0,) * S, (0,) * S, (-1,) * S, ((),) * S)
    seen = {start}
    queue = deque([start])

    def arrive(emptyk, pend, s):
        p2, e2 = list(pend), list(emptyk)
        p2[s] += 1
        if p2[s] == W:
            p2[s] = 0
            e2[s] += 1
        return tuple(e2), tuple(p2)

    while queue:
        st = queue.popleft()
        p_it, warps, fullk, emptyk, pend, content, posts = st
        nxt = []
        if p_it < B:  # producer
            s = p_it % S
            if p_it < S or not producer_waits or (emptyk[s] & 1) != (((p_it // S) - 1) & 1):
                c2 = list(content)
                c2[s] = p_it
                f2 = list(fullk)
                f2[s] += 1
                nxt.append((p_it + 1, warps, tuple(f2), emptyk, pend, tuple(c2), posts))
        for w, (it, step) in enumerate(warps):
            if it >= B:
                continue
            s = it % S
            w2 = list(warps)
            if step == 0:  # wait for the stage
                if (fullk[s] & 1) != consumer_parity(it, S):
                    w2[w] = (it, 1)
                    nxt.append((p_it, tuple(w2), fullk, emptyk, pend, content, posts))
            elif step == 1:  # read it; short blocks release it at once
                if content[s] != it:
                    return len(seen), f"warp {w} read block {content[s]} in stage {s}, expected {it}"
                if long_block(it):
                    ps = list(posts)
                    ps[s] = ps[s] + (it,)
                    w2[w] = (it, 2 if w == 0 else 3)
                    nxt.append((p_it, tuple(w2), fullk, emptyk, pend, content, tuple(ps)))
                else:
                    e2, p2 = arrive(emptyk, pend, s)
                    w2[w] = (it + 1, 0)
                    nxt.append((p_it, tuple(w2), fullk, e2, p2, content, posts))
            elif step == 2:  # warp 0 combines the partials of the block
                if len(posts[s]) >= W:  # the kernel waits while the count is below W
                    if any(t != it for t in posts[s]):
                        return len(seen), f"warp 0 combined partials of blocks {posts[s]} for block {it}"
                    ps = list(posts)
                    if reset_before_arrive:
                        ps[s] = ()
                        e2, p2 = arrive(emptyk, pend, s)
                        w2[w] = (it + 1, 0)
                    else:
                        e2, p2 = arrive(emptyk, pend, s)
                        w2[w] = (it, 4)
                    nxt.append((p_it, tuple(w2), fullk, e2, p2, content, tuple(ps)))
            elif step == 3:  # other warps release the stage after posting
                e2, p2 = arrive(emptyk, pend, s)
                w2[w] = (it + 1, 0)
                nxt.append((p_it, tuple(w2), fullk, e2, p2, content, posts))
            elif step == 4:  # (negative control) reset after the arrival
                ps = list(posts)
                ps[s] = ()
                w2[w] = (it + 1, 0)
                nxt.append((p_it, tuple(w2), fullk, emptyk, pend, content, tuple(ps)))
        if not nxt and not (p_it == B and all(it == B for it, _ in warps)):
            return len(seen), f"deadlock at producer block {p_it}, warps {warps}"
        for n in nxt:
            if n not in seen:
                seen.add(n)
                queue.append(n)
    return len(seen), None


@pytest.mark.parametrize("W,S,B", [(2, 2, 7), (3, 2, 6), (2, 3, 8), (3, 3, 7), (4, 2, 5), (2, 5, 11)])
def test_per_warp_waits_are_safe(W, S, B):
    states, bad = explore(W, S, B)
    assert bad is None, bad
    assert states > 10


def test_wrong_parity_is_caught():
    """Negative control: waiting on the block's parity instead of the stage
    use's parity lets a warp pass a phase it does not mean."""
    _, bad = explore(2, 3, 8, consumer_parity=lambda it, S: it & 1)
    assert bad is not None


def test_refill_without_empty_wait_is_caught():
    """Negative control: a producer that does not wait for the empty barrier
    overwrites a stage a warp has not finished reading."""
    _, bad = explore(2, 2, 6, producer_waits=False)
    assert bad is not None and "read block" in bad



@pytest.mark.parametrize("W,S,B", [(2, 2, 7), (3, 2, 6), (2, 3, 8), (3, 3, 7)])
def test_long_row_combine_is_safe(W, S, B):
    """Blocks alternate between ordinary rows and one long row shared by all
    warps (every block of stage 0, and every third block)."""
    states, bad = explore(W, S, B, long_block=lambda it: it % S == 0 or it % 3 == 1)
    assert bad is None, bad
    _, bad = explore(W, S, B, long_block=lambda it: True)
    assert bad is None, bad


def test_late_counter_reset_is_caught():
    """Negative control: resetting the partial counter after releasing the
    stage lets the stage's next use post before the reset, which then wipes
    that post: warp 0 waits for a partial that never comes (in the kernel its
    bounded wait runs out)."""
    _, bad = explore(2, 2, 8, long_block=lambda it: True, reset_before_arrive=False)
    assert bad is not None
