"""FP64 CPU adjoint of the 2-D Darcy column loss (TEST INFRASTRUCTURE ONLY).

The oracle for cfdrs_b200.adjoint: forward and adjoint by sparse direct
solves (scipy SuperLU), and dL/dtheta from the face-by-face adjoint formula
derived by hand -- an independent route from the device path, which
differentiates its torch assembly automatically.

System: -div(k grad p) = 0, k = exp(theta), n x n cells (row i + n*j),
harmonic-mean face coefficient k_f = 2 k_P k_E / (k_P + k_E), Dirichlet
p = 1 / p = 0 on the left / right walls at half a cell (2 k_P on the diagonal,
2 k_P * 1 in b on the left), no flux top and bottom. Loss L = sum p^2 over one
cell column. With A^T lambda = dL/dp:
  face (P, E):   dL/dk_f = -(lambda_P - lambda_E)(p_P - p_E)
  left wall P:   dL/dk_P += -2 lambda_P (p_P - 1)
  right wall P:  dL/dk_P += -2 lambda_P p_P
  dk_f/dk_P = 2 k_E^2 / (k_P + k_E)^2,   dL/dtheta_P = k_P dL/dk_P.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def assemble(theta: np.ndarray):
    """Same system as cfdrs_b200.problems.darcy_2d, assembled independently."""
    n = theta.shape[0]
    k = np.exp(theta)
    N = n * n
    idx = np.arange(N).reshape(n, n)  # [j, i]
    rows, cols, vals = [], [], []
    diag = np.zeros((n, n))

    def hm(a, b):
        return 2.0 * a * b / (a + b)

    fx = hm(k[:, :-1], k[:, 1:])
    fy = hm(k[:-1, :], k[1:, :])
    for (P, E, f) in ((idx[:, :-1], idx[:, 1:], fx), (idx[:-1, :], idx[1:, :], fy)):
        rows += [P.ravel(), E.ravel()]
        cols += [E.ravel(), P.ravel()]
        vals += [-f.ravel(), -f.ravel()]
    diag[:, :-1] += fx
    diag[:, 1:] += fx
    diag[:-1, :] += fy
    diag[1:, :] += fy
    diag[:, 0] += 2.0 * k[:, 0]
    diag[:, -1] += 2.0 * k[:, -1]
    rows.append(idx.ravel())
    cols.append(idx.ravel())
    vals.append(diag.ravel())
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    b = np.zeros((n, n))
    b[:, 0] = 2.0 * k[:, 0]
    return A, b.ravel()


def loss_and_grad(theta: np.ndarray, column: int):
    n = theta.shape[0]
    k = np.exp(theta)
    A, b = assemble(theta)
    lu = spla.splu(A.tocsc())
    p = lu.solve(b)
    P2 = p.reshape(n, n)
    L = float((P2[:, column] ** 2).sum())
    g = np.zeros((n, n))
    g[:, column] = 2.0 * P2[:, column]
    lam = lu.solve(g.ravel(), trans="T").reshape(n, n)
    dk = np.zeros((n, n))
    # x faces between (j, i) and (j, i+1)
    kP, kE = k[:, :-1], k[:, 1:]
    dLf = -(lam[:, :-1] - lam[:, 1:]) * (P2[:, :-1] - P2[:, 1:])
    dk[:, :-1] += dLf * 2.0 * kE ** 2 / (kP + kE) ** 2
    dk[:, 1:] += dLf * 2.0 * kP ** 2 / (kP + kE) ** 2
    # y faces between (j, i) and (j+1, i)
    kP, kE = k[:-1, :], k[1:, :]
    dLf = -(lam[:-1, :] - lam[1:, :]) * (P2[:-1, :] - P2[1:, :])
    dk[:-1, :] += dLf * 2.0 * kE ** 2 / (kP + kE) ** 2
    dk[1:, :] += dLf * 2.0 * kP ** 2 / (kP + kE) ** 2
    dk[:, 0] += -2.0 * lam[:, 0] * (P2[:, 0] - 1.0)
    dk[:, -1] += -2.0 * lam[:, -1] * P2[:, -1]
    return L, k * dk, p


def loss(theta: np.ndarray, column: int) -> float:
    A, b = assemble(theta)
    p = spla.splu(A.tocsc()).solve(b)
    return float((p.reshape(theta.shape)[:, column] ** 2).sum())


def central_fd(theta: np.ndarray, column: int, cells, h: float = 1e-6):
    """Central differences (L(theta + h e_c) - L(theta - h e_c)) / 2h, FP64 direct solves."""
    out = []
    for (j, i) in cells:
        tp = theta.copy()
        tp[j, i] += h
        tm = theta.copy()
        tm[j, i] -= h
        out.append((loss(tp, column) - loss(tm, column)) / (2.0 * h))
    return np.array(out)


def central_fd_lowrank(theta: np.ndarray, column: int, cells, h: float = 1e-6):
    """The same central differences as central_fd, with every perturbed system
    solved from ONE sparse LU of the unperturbed A: perturbing theta at one
    cell changes A only on the rows and columns S of that cell and its (at
    most 4) neighbours, A' = A + E_S M E_S^T with M = (A' - A)[S, S], so by the
    Woodbury identity
        A'^-1 b' = y - Z M (I + Z_S M)^-1 y_S,  y = A^-1 b',  Z = A^-1 E_S,
    (Z_S, y_S: the rows S of Z and y). Exact algebra, |S| + 2 triangular solve
    pairs per cell instead of two factorizations."""
    n = theta.shape[0]
    A, b = assemble(theta)
    lu = spla.splu(A.tocsc())
    out = []
    for (j, i) in cells:
        S = [j * n + i]
        for dj, di in ((-1, 0), (1, 0), (0, -1), (0, 1)):
            jj, ii = j + dj, i + di
            if 0 <= jj < n and 0 <= ii < n:
                S.append(jj * n + ii)
        S = np.array(S)
        E = np.zeros((n * n, S.size))
        E[S, np.arange(S.size)] = 1.0
        Z = lu.solve(E)
        vals = []
        for sgn in (1.0, -1.0):
            t = theta.copy()
            t[j, i] += sgn * h
            A2, b2 = assemble(t)
            M = (A2 - A)[S][:, S].toarray()
            y = lu.solve(b2)
            K = np.eye(S.size) + Z[S, :] @ M
            p = y - Z @ (M @ np.linalg.solve(K, y[S]))
            vals.append(float((p.reshape(n, n)[:, column] ** 2).sum()))
        out.append((vals[0] - vals[1]) / (2.0 * h))
    return np.array(out)
