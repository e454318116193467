"""The storage scheme of the device Gauss-Jordan coarse inverse (k_gj_coop in
cfdrs_b200/csrc/recompute.cu), modelled step for step in numpy and compared
with the host algorithm (dense_inverse in amg_setup.cpp: pivot = first row of
largest |m[r][c]| for r >= c, swap, scale the pivot row by 1/m[c][c],
row_r -= m[r][c] row_c for every other row with m[r][c] != 0).

The model keeps what the kernel keeps: rows of n + 1 entries holding the
inverse columns already in use followed by the live columns of the eliminated
matrix (unit inverse columns are not stored), rows reached through a table of
physical buffers with two spares (a swap is a table update), the per-step
argmax of the next column taken from the updated rows, and the final scatter
by the pivots' original row numbers. Numpy's elementwise float64 operations
round each product and difference separately, as the kernel's __dmul_rn /
__dsub_rn do, so equality is exact."""
import numpy as np
import pytest


def host_gauss_jordan(A):
    n = A.shape[0]
    m = A.copy()
    inv = np.eye(n)
    for c in range(n):
        p = c
        for r in range(c + 1, n):
            if abs(m[r, c]) > abs(m[p, c]):
                p = r
        if m[p, c] == 0.0:
            return None
        if p != c:
            m[[c, p]] = m[[p, c]]
            inv[[c, p]] = inv[[p, c]]
        d = 1.0 / m[c, c]
        m[c] *= d
        inv[c] *= d
        for r in range(n):
            if r == c:
                continue
            f = m[r, c]
            if f == 0.0:
                continue
            m[r] -= f * m[c]
            inv[r] -= f * inv[c]
    return inv


def table_gauss_jordan(A):
    n = A.shape[0]
    ldw = (n + 2) & ~1
    W = np.zeros((n + 2, ldw))
    W[:n, 1:n + 1] = A           # slot 0 unused at first; m[r][k] at slot k + 1
    phys = list(range(n))        # logical row -> physical buffer
    orig = list(range(n))        # logical row -> original row (owner of its unit column)
    spare = [n, n + 1]
    qcol = [0] * n               # original row of step j's pivot

    def argmax(cands):
        bv, br = -1.0, n
        for v, r in cands:
            if v > bv or (v == bv and r < br):
                bv, br = v, r
        return bv, br

    bv, br = argmax([(abs(W[r, 1]), r) for r in range(n)])
    for c in range(n):
        if not bv > 0.0:
            return None
        p = br
        Wp, Wc = W[phys[p]].copy(), W[phys[c]].copy()
        d = 1.0 / Wp[c + 1]
        PW = np.array([d if j == c else Wp[j] * d for j in range(ldw)])
        new_rows, cands = {}, []
        for r in range(n):
            if r == c:
                new_rows[spare[0]] = PW[:n + 1].copy()
                continue
            moved = r == p
            src = Wc if moved else W[phys[r]]
            dst = spare[1] if moved else phys[r]
            f = src[c + 1]
            row = src[:n + 1].copy()
            row[c] = 0.0                     # the pivot's unit column enters at slot c
            if f != 0.0:
                row = row - f * PW[:n + 1]
            new_rows[dst] = row
            if c + 1 < n and r > c:
                cands.append((abs(row[c + 2]), r))
        for k, v in new_rows.items():
            W[k, :n + 1] = v
        oc, op = phys[c], phys[p]
        phys[c] = spare[0]
        if p != c:
            phys[p] = spare[1]
            spare[1] = op
            orig[c], orig[p] = orig[p], orig[c]
        spare[0] = oc
        qcol[c] = orig[c]
        if c + 1 < n:
            bv, br = argmax(cands)
    inv = np.zeros((n, n))
    for r in range(n):
        for j in range(n):
            inv[r, qcol[j]] = W[phys[r], j]
    return inv


@pytest.mark.parametrize("trial", range(24))
def test_table_scheme_reproduces_host_gauss_jordan(trial):
    rng = np.random.default_rng(trial)
    n = int(rng.integers(1, 32))
    A = np.where(rng.uniform(size=(n, n)) < rng.uniform(0.05, 0.6), rng.uniform(-1, 1, (n, n)), 0.0)
    if trial % 3 == 0:
        A += 3.0 * np.eye(n)                 # diagonally dominant: few row exchanges
    if trial % 5 == 1:
        A = A[rng.permutation(n)]            # permuted: exchanges at most pivots
    host, table = host_gauss_jordan(A), table_gauss_jordan(A)
    assert (host is None) == (table is None)  # singular in both or in neither
    if host is not None:
        assert np.array_equal(host.view(np.int64), table.view(np.int64))  # bit for bit
