"""Exhaustive check of the cross-CTA synchronisation of the cooperative
Gauss-Jordan coarse inverse (k_gj_coop in cfdrs_b200/csrc/recompute.cu): G CTAs
take N pivot steps with one grid barrier per step. Every interleaving of the
model is explored (breadth first).

Per step c every CTA: reads all CTAs' argmax partials for column c (one of two
buffers, by step parity); reads the pivot row p and row c from their physical
buffers; rewrites its own rows (row c into spare 0, row p into spare 1, the
rest in place); updates its copy of the row table (the old buffers of rows c
and p become the spares); writes its partial for column c + 1 into the other
buffer; arrives on the barrier counter and waits for (c + 2) G arrivals.

Every buffer and partial write is tagged with its step; a read must find the
tag it means (rows written in step c - 1, partials for column c). Checked
over pivot sequences with and without row exchanges; a single partial buffer
and rows written in place (no spares) are each caught (negative controls)."""
from collections import deque

import pytest


def explore(G, N, pivots, double_buffer=True, spares=True):
    """pivots[c] = the pivot row of step c (>= c). Returns (states, violation)."""
    n = N
    INIT = -1

    def program(g):
        """The CTA's actions, each applied atomically."""
        ops = [("post", 0), ("arrive",), ("wait", G)]
        for c in range(N):
            ops.append(("read_partials", c))
            ops.append(("read_pivot_rows", c))
            for r in range(g, n, G):
                ops.append(("row", c, r))
            ops.append(("table", c))
            if c + 1 < N:
                ops.append(("post", c + 1))
            ops.append(("arrive",))
            ops.append(("wait", (c + 2) * G))
        return ops

    progs = [program(g) for g in range(G)]
    # shared: buffer tags (n + 2 buffers), partial tags [2][G], barrier count
    # per CTA: program counter, row table (logical -> physical), spares
    start_tables = tuple((tuple(range(n)), (n, n + 1)) for _ in range(G))
    start = ((0,) * G, start_tables, (INIT,) * n + (None, None), ((None,) * G, (None,) * G), 0)
    seen = {start}
    queue = deque([start])
    while queue:
        st = queue.popleft()
        pcs, tables, bufs, parts, count = st
        moves = []
        for g in range(G):
            if pcs[g] >= len(progs[g]):
                continue
            op = progs[g][pcs[g]]
            phys, spare = tables[g]
            kind = op[0]
            new_bufs, new_parts, new_count, new_table = bufs, parts, count, tables[g]
            if kind == "wait":
                if count < op[1]:
                    continue
            elif kind == "arrive":
                new_count = count + 1
            elif kind == "post":
                slot = (op[1] & 1) if double_buffer else 0
                ps = [list(parts[0]), list(parts[1])]
                ps[slot][g] = op[1]
                new_parts = (tuple(ps[0]), tuple(ps[1]))
            elif kind == "read_partials":
                c = op[1]
                slot = (c & 1) if double_buffer else 0
                if any(t != c for t in parts[slot]):
                    return len(seen), f"CTA {g} step {c} read partials {parts[slot]}"
            elif kind == "read_pivot_rows":
                c = op[1]
                want = c - 1 if c > 0 else INIT
                for r in (pivots[c], c):
                    if bufs[phys[r]] != want:
                        return len(seen), f"CTA {g} step {c} read row {r} tagged {bufs[phys[r]]}"
            elif kind == "row":
                c, r = op[1], op[2]
                want = c - 1 if c > 0 else INIT
                p = pivots[c]
                b = list(bufs)
                if r == c:
                    b[spare[0] if spares else phys[r]] = c
                elif r == p:
                    b[spare[1] if spares else phys[r]] = c
                else:
                    if bufs[phys[r]] != want:
                        return len(seen), f"CTA {g} step {c} updated row {r} tagged {bufs[phys[r]]}"
                    b[phys[r]] = c
                new_bufs = tuple(b)
            elif kind == "table":
                c = op[1]
                p = pivots[c]
                if spares:
                    ph, sp = list(phys), list(spare)
                    oc, op_ = ph[c], ph[p]
                    ph[c] = sp[0]
                    if p != c:
                        ph[p] = sp[1]
                        sp[1] = op_
                    sp[0] = oc
                    new_table = (tuple(ph), tuple(sp))
                else:
                    ph = list(phys)
                    ph[c], ph[p] = ph[p], ph[c]
                    new_table = (tuple(ph), spare)
            pc2 = list(pcs)
            pc2[g] += 1
            t2 = list(tables)
            t2[g] = new_table
            moves.append((tuple(pc2), tuple(t2), new_bufs, new_parts, new_count))
        if not moves and any(pcs[g] < len(progs[g]) for g in range(G)):
            return len(seen), f"deadlock: program counters {pcs}, barrier count {count}"
        for m in moves:
            if m not in seen:
                seen.add(m)
                queue.append(m)
    return len(seen), None


PIVOTS = {
    "no_exchange": lambda N: list(range(N)),
    "next_row": lambda N: [min(c + 1, N - 1) for c in range(N)],
    "last_row": lambda N: [N - 1] * N,
    "mixed": lambda N: [N - 1 if c % 2 == 0 else c for c in range(N)],
}


@pytest.mark.parametrize("G,N", [(2, 3), (2, 4), (3, 3)])
@pytest.mark.parametrize("pattern", sorted(PIVOTS))
def test_one_barrier_per_step_is_safe(G, N, pattern):
    states, bad = explore(G, N, PIVOTS[pattern](N))
    assert bad is None, bad
    assert states > 20


def test_single_partial_buffer_is_caught():
    """A CTA that finishes a step while another has not yet read that step's
    partials would overwrite them."""
    _, bad = explore(2, 3, PIVOTS["mixed"](3), double_buffer=False)
    assert bad is not None and "partials" in bad


def test_rows_in_place_are_caught():
    """Writing the new pivot row into the buffer the other CTAs read it from
    races with their reads of the same step."""
    _, bad = explore(2, 3, PIVOTS["mixed"](3), spares=False)
    assert bad is not None
