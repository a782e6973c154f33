"""P2 nodal operators on the reference triangle, restated from the published algorithms.

The reference ships these as text files produced offline by MATLAB
(precompute_matrices_with_matlab/precompute_matrices.m:14-44): the Vandermonde matrix ``V`` of
the orthonormal Dubiner basis at the six P2 nodes, its inverse, the gradient Vandermonde
matrices ``Vr``/``Vs``, the 1D face Vandermonde ``Vb`` and the three face lift matrices
``S1..S3 = V Vib_j^T inv(Vb)^T inv(Vb)``.  The basis functions follow Hesthaven & Warburton,
*Nodal Discontinuous Galerkin Methods* (2008), sections 3.1 and 6.1 (JacobiP, Simplex2DP,
GradSimplex2DP); the nodes are the P2 "Fekete" set of Fekete_Degree2.m:2-9 (three vertices and
three edge midpoints) mapped to [-1,1]^2 (precompute_matrices.m:10-11).

MATLAB stores them with ``save -ascii`` at 8 significant digits; ``to_text`` reproduces that
format so the same reader parses both.
"""
from __future__ import annotations

import math

import numpy as np

N = 2
NP = 6
NFP = 3

# Fekete_Degree2.m:2-9 on [0,1]^2, mapped by 2*x - 1 (precompute_matrices.m:10-11)
_FEKETE01 = np.array([[1.0, 0.0], [0.5, 0.5], [0.0, 1.0], [0.5, 0.0], [0.0, 0.5], [0.0, 0.0]])
FEKETE = 2.0 * _FEKETE01 - 1.0

# Face node lists, 1-based, face 0 = v0->v1, 1 = v1->v2, 2 = v0->v2 (fun_DG.c:1046-1057)
IBE = np.array([[6, 4, 1], [1, 2, 3], [6, 5, 3]], dtype=np.int64)


def jacobi_p(x: np.ndarray, alpha: float, beta: float, n: int) -> np.ndarray:
    """Orthonormal Jacobi polynomial P_n^(alpha,beta)(x) by the three-term recurrence."""
    x = np.asarray(x, dtype=np.float64)
    pl = np.zeros((n + 1, x.size))
    g0 = 2.0 ** (alpha + beta + 1) / (alpha + beta + 1) * math.gamma(alpha + 1) * \
        math.gamma(beta + 1) / math.gamma(alpha + beta + 1)
    pl[0] = 1.0 / math.sqrt(g0)
    if n == 0:
        return pl[0].copy()
    g1 = (alpha + 1) * (beta + 1) / (alpha + beta + 3) * g0
    pl[1] = ((alpha + beta + 2) * x / 2 + (alpha - beta) / 2) / math.sqrt(g1)
    if n == 1:
        return pl[1].copy()
    aold = 2.0 / (2 + alpha + beta) * math.sqrt((alpha + 1) * (beta + 1) / (alpha + beta + 3))
    for i in range(1, n):
        h1 = 2 * i + alpha + beta
        anew = 2.0 / (h1 + 2) * math.sqrt((i + 1) * (i + 1 + alpha + beta) * (i + 1 + alpha) *
                                          (i + 1 + beta) / (h1 + 1) / (h1 + 3))
        bnew = -(alpha * alpha - beta * beta) / h1 / (h1 + 2)
        pl[i + 1] = 1.0 / anew * (-aold * pl[i - 1] + (x - bnew) * pl[i])
        aold = anew
    return pl[n].copy()


def grad_jacobi_p(x: np.ndarray, alpha: float, beta: float, n: int) -> np.ndarray:
    x = np.asarray(x, dtype=np.float64)
    if n == 0:
        return np.zeros(x.size)
    return math.sqrt(n * (n + alpha + beta + 1)) * jacobi_p(x, alpha + 1, beta + 1, n - 1)


def _rs_to_ab(r: np.ndarray, s: np.ndarray):
    a = np.where(s != 1.0, 2.0 * (1.0 + r) / np.where(s != 1.0, 1.0 - s, 1.0) - 1.0, -1.0)
    return a, s.copy()


def _simplex2dp(a, b, i, j):
    return math.sqrt(2.0) * jacobi_p(a, 0, 0, i) * jacobi_p(b, 2 * i + 1, 0, j) * (1 - b) ** i


def _grad_simplex2dp(a, b, i, j):
    fa = jacobi_p(a, 0, 0, i)
    dfa = grad_jacobi_p(a, 0, 0, i)
    gb = jacobi_p(b, 2 * i + 1, 0, j)
    dgb = grad_jacobi_p(b, 2 * i + 1, 0, j)
    dr = dfa * gb
    if i > 0:
        dr = dr * (0.5 * (1 - b)) ** (i - 1)
    ds = dfa * (gb * (0.5 * (1 + a)))
    if i > 0:
        ds = ds * (0.5 * (1 - b)) ** (i - 1)
    tmp = dgb * (0.5 * (1 - b)) ** i
    if i > 0:
        tmp = tmp - 0.5 * i * gb * (0.5 * (1 - b)) ** (i - 1)
    ds = ds + fa * tmp
    return dr * 2.0 ** (i + 0.5), ds * 2.0 ** (i + 0.5)


def vandermonde2d(n: int, r: np.ndarray, s: np.ndarray) -> np.ndarray:
    a, b = _rs_to_ab(r, s)
    cols = [_simplex2dp(a, b, i, j) for i in range(n + 1) for j in range(n - i + 1)]
    return np.stack(cols, 1)


def grad_vandermonde2d(n: int, r: np.ndarray, s: np.ndarray):
    a, b = _rs_to_ab(r, s)
    pairs = [_grad_simplex2dp(a, b, i, j) for i in range(n + 1) for j in range(n - i + 1)]
    return np.stack([p[0] for p in pairs], 1), np.stack([p[1] for p in pairs], 1)


def vandermonde1d(n: int, r: np.ndarray) -> np.ndarray:
    return np.stack([jacobi_p(r, 0, 0, j) for j in range(n + 1)], 1)


def p2_operators() -> dict:
    """Exact (double precision) P2 operators in the layout of the shipped text files."""
    r, s = FEKETE[:, 0], FEKETE[:, 1]
    V = vandermonde2d(N, r, s)
    inverV = np.linalg.inv(V)
    Vr, Vs = grad_vandermonde2d(N, r, s)
    edge1 = FEKETE[[5, 3, 0]]
    Vb = vandermonde1d(N, edge1[:, 0])
    inverVb = np.linalg.inv(Vb)
    out = {"FeketeNew": FEKETE.copy(), "V": V, "inverV": inverV, "Vr": Vr, "Vs": Vs,
           "Vb": Vb, "inverVb": inverVb}
    for name, rows in (("S1", [5, 3, 0]), ("S2", [0, 1, 2]), ("S3", [5, 4, 2])):
        vib = V[rows]
        out[name] = V @ vib.T @ inverVb.T @ inverVb
    return out


SHAPES = {"FeketeNew": (NP, 2), "S1": (NP, 3), "S2": (NP, 3), "S3": (NP, 3), "V": (NP, NP),
          "Vb": (3, 3), "Vr": (NP, NP), "Vs": (NP, NP), "inverV": (NP, NP), "inverVb": (3, 3)}


def to_text(m: np.ndarray) -> str:
    """MATLAB ``save -ascii`` rendering (``%16.7e`` per value)."""
    return "".join("".join("%16.7e" % v for v in row) + "\n" for row in np.atleast_2d(m))


def write_text_files(directory: str, ops: dict | None = None) -> None:
    """Write the ten ``*.txt`` operator files the reference driver reads (DG_leap_Frog_OpenMP.c:65-94)."""
    import os
    ops = p2_operators() if ops is None else ops
    os.makedirs(directory, exist_ok=True)
    for name in SHAPES:
        with open(os.path.join(directory, name + ".txt"), "w") as f:
            f.write(to_text(ops[name]))
