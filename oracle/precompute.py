"""Restatement of ScalFMM's symmetric-compressed M2L operator precompute, in numpy.

TEST INFRASTRUCTURE ONLY: the checker for the product's own FP64 operator compression.

Follows ``precompute`` in Src/Kernels/Chebyshev/FChebSymM2LHandler.hpp:39-281 (paths relative to the
reference project root):

* the 16 canonical transfer vectors (i, j, k), 2 <= i <= 3, 0 <= k <= j <= i, with source cells of
  reference width 2 centred at 2*(i, j, k) (:76-81);
* the weighted kernel matrix A[t, s] = w_t w_s / |X_t - Y_s| (EntryComputer,
  Src/Kernels/Interpolation/FInterpMatrixKernel.hpp:561-600; root-of-weights
  Src/Kernels/Chebyshev/FChebTensor.hpp:42-55);
* partially pivoted ACA (FAca::pACA, Src/Utils/FAca.hpp:141-225);
* QR of both factors, SVD of Ru Rv^T, rank by FSvd::getRank (Src/Utils/FSvd.hpp:53-64) (:131-206);
* un-weighting of the rows (:257-261).
"""
from __future__ import annotations

import numpy as np


def cheb_roots(order: int) -> np.ndarray:
    """Ascending Chebyshev roots (FChebRoots.hpp:31-36)."""
    j = np.arange(order)
    return -np.cos(np.pi * (2 * j + 1) / (2 * order))


def node_coords(roots: np.ndarray, center, width: float) -> np.ndarray:
    """Interpolation nodes of a cell (FInterpTensor::setRoots, FInterpTensor.hpp:70-84); node id
    n = nx + p*ny + p*p*nz."""
    p = len(roots)
    n = np.arange(p ** 3)
    loc = np.stack([roots[n % p], roots[(n // p) % p], roots[n // (p * p)]], axis=1)
    return np.asarray(center, dtype=np.float64)[None, :] + 0.5 * width * loc


def root_of_weights(order: int) -> np.ndarray:
    """sqrt of the tensor Chebyshev quadrature weights (FChebTensor::setRootOfWeights)."""
    r = cheb_roots(order)
    w1 = np.pi / order * np.sqrt(1.0 - r * r)
    p = order
    n = np.arange(p ** 3)
    return np.sqrt(w1[n % p] * w1[(n // p) % p] * w1[n // (p * p)])


def paca(row, col, nx: int, ny: int, eps: float):
    """Partially pivoted ACA, FAca.hpp:141-225.  row(I) returns A[I, :], col(J) returns A[:, J]."""
    r_free = np.ones(nx, dtype=bool)
    c_free = np.ones(ny, dtype=bool)
    U, V = [], []
    norm2S = 0.0
    I = 0
    J = 0
    eps2 = eps * eps
    while True:
        v = row(I).copy()
        r_free[I] = False
        for u_l, v_l in zip(U, V):
            v -= u_l[I] * v_l
        a = np.abs(v)
        best = 0.0
        for j in range(ny):  # first strict maximum among unused columns, as the reference scans
            if c_free[j] and best < a[j]:
                best = a[j]
                J = j
        v = v * (1.0 / v[J])
        u = col(J).copy()
        c_free[J] = False
        for u_l, v_l in zip(U, V):
            u -= v_l[J] * u_l
        a = np.abs(u)
        best = 0.0
        for i in range(nx):
            if r_free[i] and best < a[i]:
                best = a[i]
                I = i
        cross = 0.0
        for u_l, v_l in zip(U, V):
            cross += float(u @ u_l) * float(v_l @ v)
        norm2uv = float(u @ u) * float(v @ v)
        norm2S += norm2uv + 2.0 * cross
        U.append(u)
        V.append(v)
        if not norm2uv > eps2 * norm2S:
            break
    return np.stack(U, axis=1), np.stack(V, axis=1)


def get_rank(s: np.ndarray, eps: float) -> int:
    """FSvd::getRank: smallest k with sum_{i>=k} s_i^2 <= eps^2 sum s_i^2 (scanning from the tail)."""
    nrm2 = float(s @ s)
    acc = 0.0
    for k in range(len(s), 0, -1):
        acc += s[k - 1] * s[k - 1]
        if acc > eps * eps * nrm2:
            return k
    raise RuntimeError("rank cannot be larger than size")


def class_slots():
    out = []
    for i in (2, 3):
        for j in range(0, i + 1):
            for k in range(0, j + 1):
                out.append(((i + 3) * 49 + (j + 3) * 7 + (k + 3), (i, j, k)))
    return out


def sym_operators(order: int, eps: float | None = None):
    """Return {slot: (U, V)} with U, V of shape (p^3, r): K(X_n, Y_m) ~ sum_r U[n, r] V[m, r]."""
    if eps is None:
        eps = 10.0 ** (-order)
    roots = cheb_roots(order)
    X = node_coords(roots, (0.0, 0.0, 0.0), 2.0)
    w = root_of_weights(order)
    nn = order ** 3
    ops = {}
    for slot, (i, j, k) in class_slots():
        Y = node_coords(roots, (2.0 * i, 2.0 * j, 2.0 * k), 2.0)

        def row(I, X=X, Y=Y):
            d = X[I][None, :] - Y
            return w[I] * w / np.sqrt((d * d).sum(1))

        def col(J, X=X, Y=Y):
            d = X - Y[J][None, :]
            return w * w[J] / np.sqrt((d * d).sum(1))

        UU, VV = paca(row, col, nn, nn, eps)
        Qu, Ru = np.linalg.qr(UU)
        Qv, Rv = np.linalg.qr(VV)
        phi = Ru @ Rv.T
        Ur, s, VrT = np.linalg.svd(phi)
        r = get_rank(s, eps)
        U = Qu @ (Ur[:, :r] * s[:r][None, :])
        V = Qv @ VrT[:r, :].T
        U = U / w[:, None]
        V = V / w[:, None]
        ops[slot] = (U, V)
    return ops


def pack_reference_layout(ops: dict, order: int):
    """ranks[343] and the packed U|V buffer in the reference's storage order (FChebSymM2LHandler.hpp:
    183-203: U column-major then V column-major, slots in increasing order)."""
    nn = order ** 3
    ranks = np.zeros(343, dtype=np.int32)
    chunks = []
    for slot in sorted(ops):
        U, V = ops[slot]
        ranks[slot] = U.shape[1]
        chunks.append(np.asfortranarray(U).reshape(-1, order="F"))
        chunks.append(np.asfortranarray(V).reshape(-1, order="F"))
    assert all(c.size % nn == 0 for c in chunks)
    return ranks, np.concatenate(chunks).astype(np.float64)
