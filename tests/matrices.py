"""Seeded test matrices in CSC form (0-based, rows ascending per column)."""
from __future__ import annotations

import numpy as np


def csc_from_dense_pattern(A, pat):
    n = A.shape[0]
    cols = [np.nonzero(pat[:, j])[0] for j in range(n)]
    cp = np.zeros(n + 1, np.int32)
    cp[1:] = np.cumsum([len(c) for c in cols])
    ri = np.concatenate(cols).astype(np.int32) if n else np.zeros(0, np.int32)
    vals = np.concatenate([A[c, j] for j, c in enumerate(cols)]).astype(np.float64)
    return n, cp, ri, vals


def random_matrix(rng, n, density, diag_dominant=True, zero_diag_frac=0.0, integer=False):
    """Random sparse matrix; some diagonals structurally absent when
    zero_diag_frac > 0 (forces off-diagonal and singleton pivots)."""
    A = (rng.random((n, n)) < density) * rng.standard_normal((n, n))
    if integer:
        A = np.round(A * 2)
    if diag_dominant:
        np.fill_diagonal(A, np.abs(A).sum(1) + 1.0)
    kill = rng.random(n) < zero_diag_frac
    A[kill, kill] = 0
    pat = (A != 0) | (np.eye(n, dtype=bool) & ~np.diag(kill))
    for i in range(n):
        if not pat[i].any() or not pat[:, i].any():
            pat[i, i] = True
            A[i, i] = 1.0
    return csc_from_dense_pattern(A, pat)


def mna_mesh(rng, side, n_vsrc=1, r_sigma=0.1):
    """Resistor mesh MNA matrix with voltage-source branch rows (+-1 twins)."""
    N = side * side
    ent = {}

    def add(r, c, v):
        ent[(r, c)] = ent.get((r, c), 0.0) + v

    for y in range(side):
        for x in range(side):
            i = y * side + x
            for (xx, yy) in ((x + 1, y), (x, y + 1)):
                if xx < side and yy < side:
                    j = yy * side + xx
                    g = 1.0 / (1000.0 * np.exp(r_sigma * rng.standard_normal()))
                    add(i, i, g)
                    add(j, j, g)
                    add(i, j, -g)
                    add(j, i, -g)
    n = N + n_vsrc
    nodes = rng.choice(N, size=n_vsrc, replace=False)
    for k, node in enumerate(nodes):
        b = N + k
        add(int(node), b, 1.0)
        add(b, int(node), 1.0)
    keys = sorted(ent, key=lambda rc: (rc[1], rc[0]))
    cp = np.zeros(n + 1, np.int32)
    for (_, c) in keys:
        cp[c + 1] += 1
    cp = np.cumsum(cp).astype(np.int32)
    ri = np.array([r for r, _ in keys], np.int32)
    vals = np.array([ent[k] for k in keys])
    return n, cp, ri, vals


def banded(n, bw=7, seed=0):
    """Diagonally dominant banded matrix in the shape of the reference's
    solver benchmark (bandwidth 7)."""
    rng = np.random.default_rng(seed)
    A = np.zeros((n, n))
    for i in range(n):
        for j in range(max(0, i - bw // 2), min(n, i + bw // 2 + 1)):
            if i != j:
                A[i, j] = -rng.uniform(0.1, 1.0)
        A[i, i] = np.abs(A[i]).sum() + 1.0
    return csc_from_dense_pattern(A, A != 0)


def dense_to_csc(A):
    A = np.asarray(A, np.float64)
    return csc_from_dense_pattern(A, np.ones_like(A, dtype=bool))


def matvec(n, cp, ri, vals, x, transposed=False):
    y = np.zeros(n)
    for j in range(n):
        for p in range(cp[j], cp[j + 1]):
            if transposed:
                y[j] += vals[p] * x[ri[p]]
            else:
                y[ri[p]] += vals[p] * x[j]
    return y
