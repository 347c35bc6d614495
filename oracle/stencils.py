"""Finite-difference stencil coefficient builders (oracle restatement).

Restates the coefficient/offset construction of gpaw/fd_operators.py; returns
plain (coef_p, offset_pc) arrays.  Test infrastructure only.
"""
from math import factorial as fact

import numpy as np

# Chelikowsky et al. Laplacian expansion, gpaw/fd_operators.py:21-28
LAPLACE = [[0],
           [-2, 1],
           [-5 / 2, 4 / 3, -1 / 12],
           [-49 / 18, 3 / 2, -3 / 20, 1 / 90],
           [-205 / 72, 8 / 5, -1 / 5, 8 / 315, -1 / 560],
           [-5269 / 1800, 5 / 3, -5 / 21, 5 / 126, -5 / 1008, 1 / 3150],
           [-5369 / 1800, 12 / 7, -15 / 56, 10 / 189, -1 / 112, 2 / 1925,
            -1 / 16632]]


def guc_laplace(gd, scale=1.0, n=1):
    """gpaw/fd_operators.py:158-204 (GUCLaplace)."""
    M_ic = np.indices((3, 3, 3)).reshape((3, -3)).T[-13:] - 1
    u_cv = gd.h_cv / (gd.h_cv ** 2).sum(1)[:, np.newaxis] ** 0.5
    u2_i = (np.dot(M_ic, u_cv) ** 2).sum(1)
    i_d = u2_i.argsort()
    m_mv = np.array([(2, 0, 0), (0, 2, 0), (0, 0, 2),
                     (0, 1, 1), (1, 0, 1), (1, 1, 0)])
    for D in range(3, 7):
        h_dv = np.dot(M_ic[i_d[:D]], gd.h_cv)
        A_md = (h_dv ** m_mv[:, np.newaxis, :]).prod(2)
        a_d, residual, rank, s = np.linalg.lstsq(A_md, [1, 1, 1, 0, 0, 0],
                                                 rcond=-1)
        if residual.sum() < 1e-14:
            if rank != D:
                raise ValueError('You have a weird unit cell!')
            break
    a_d *= scale
    offsets = [(0, 0, 0)]
    coefs = [LAPLACE[n][0] * a_d.sum()]
    for d in range(D):
        M_c = M_ic[i_d[d]]
        offsets.extend(np.arange(1, n + 1)[:, np.newaxis] * M_c)
        coefs.extend(a_d[d] * np.array(LAPLACE[n][1:]))
        offsets.extend(np.arange(-1, -n - 1, -1)[:, np.newaxis] * M_c)
        coefs.extend(a_d[d] * np.array(LAPLACE[n][1:]))
    return np.array(coefs, float), np.array(offsets, int).reshape(-1, 3)


def gradient(gd, v, scale=1.0, n=1):
    """gpaw/fd_operators.py:126-148 (Gradient)."""
    h = (gd.h_cv ** 2).sum(1) ** 0.5
    d = gd.xxxiucell_cv[:, v]
    A = np.zeros((2 * n + 1, 2 * n + 1))
    for i, io in enumerate(range(-n, n + 1)):
        for j in range(2 * n + 1):
            A[i, j] = io ** j / float(fact(j))
    A[n, 0] = 1.0
    coefs = np.linalg.inv(A)[1]
    coefs = np.delete(coefs, len(coefs) // 2)
    offs = np.delete(np.arange(-n, n + 1), n)
    coef_p = []
    offset_pc = []
    for i in range(3):
        if abs(d[i]) > 1e-11:
            coef_p.extend(list(coefs * d[i] / h[i] * scale))
            offset = np.zeros((2 * n, 3), int)
            offset[:, i] = offs
            offset_pc.extend(offset)
    return np.array(coef_p, float), np.array(offset_pc, int).reshape(-1, 3)


def laplace_A(gd, scale):
    """gpaw/fd_operators.py:211-236 (Mehrstellen A)."""
    c = np.divide(-1 / 12, gd.h_cv.diagonal() ** 2) * scale
    c0 = c[1] + c[2]
    c1 = c[0] + c[2]
    c2 = c[1] + c[0]
    a = -16.0 * np.sum(c)
    b = 10.0 * c + 0.125 * a
    coefs = [a, b[0], b[0], b[1], b[1], b[2], b[2],
             c0, c0, c0, c0, c1, c1, c1, c1, c2, c2, c2, c2]
    offsets = [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0),
               (0, 0, -1), (0, 0, 1),
               (0, -1, -1), (0, -1, 1), (0, 1, -1), (0, 1, 1),
               (-1, 0, -1), (-1, 0, 1), (1, 0, -1), (1, 0, 1),
               (-1, -1, 0), (-1, 1, 0), (1, -1, 0), (1, 1, 0)]
    return np.array(coefs, float), np.array(offsets, int)


def laplace_B(gd):
    """gpaw/fd_operators.py:239-251 (Mehrstellen B)."""
    a = 0.5
    b = 1.0 / 12.0
    coefs = [a, b, b, b, b, b, b]
    offsets = [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0),
               (0, 0, -1), (0, 0, 1)]
    return np.array(coefs, float), np.array(offsets, int)


def operator_layout(offset_pc, n_c):
    """Padding and linear offsets of gpaw/fd_operators.py:37-52.

    Returns (mp, offset_p, cfd): the uniform padding ``mp`` (the largest
    positive offset over all axes), the linear offsets into the array padded
    by ``mp`` on all six faces, and whether the stencil is a central (star)
    stencil with every offset on one axis.
    """
    offset_pc = np.asarray(offset_pc, int).reshape(-1, 3)
    cfd = True
    for offset_c in offset_pc:
        if sum([offset != 0 for offset in offset_c]) >= 2:
            cfd = False
    maxoffset_c = [max([offset_c[c] for offset_c in offset_pc])
                   for c in range(3)]
    mp = maxoffset_c[0]
    if maxoffset_c[1] != mp or maxoffset_c[2] != mp:
        mp = max(maxoffset_c)
    M_c = np.asarray(n_c) + 2 * mp
    stride_c = np.array([M_c[1] * M_c[2], M_c[2], 1])
    offset_p = np.dot(offset_pc, stride_c)
    return int(mp), np.ascontiguousarray(offset_p, dtype=np.int64), cfd
