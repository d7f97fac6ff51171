"""CPU oracle of the learned support proposal (TEST INFRASTRUCTURE ONLY: the
checker for tests/; the product library never imports it).

The network of the library's learned OMP form (include/ksvd_sm100.h,
"learned support proposal"): x = (y - mean) sqrt(n) / |y - mean|, two hidden
layers of 512
GELU units, one score per atom, binary cross-entropy between the sigmoid
scores and the OMP support mask, mean over the B x K entries.  Parameters in
the library's order: W1 [512 x n], b1, W2 [512 x 512], b2, W3 [K x 512], b3.

The reference has no counterpart (its OMP scores every atom,
cublas_matrix_omp.cu:193-233); what the proposal narrows is that pursuit,
restated here as ``omp_restricted`` (argmax of |D^T r| over the candidates
only, lowest atom index on ties, least squares on the support, the
reference's stopping rules).

Everything is float64.  With ``emulate=True`` the values the GPU keeps in
BF16 (input, weights, hidden activations, the back-propagated gradients of
the pre-activations) are rounded to BF16 (round to nearest even) at the same
points, so the GPU's gradients can be compared with it closely.
"""

from __future__ import annotations

import numpy as np
from scipy.special import erf

HIDDEN = 512


def bf16(x) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def num_params(n: int, K: int) -> int:
    return HIDDEN * n + HIDDEN + HIDDEN * HIDDEN + HIDDEN + K * HIDDEN + K


def unpack(params: np.ndarray, n: int, K: int):
    p = np.asarray(params, np.float64)
    o = 0
    out = []
    for shape in ((HIDDEN, n), (HIDDEN,), (HIDDEN, HIDDEN), (HIDDEN,), (K, HIDDEN), (K,)):
        size = int(np.prod(shape))
        out.append(p[o:o + size].reshape(shape))
        o += size
    assert o == p.size
    return out


def inputs(Y: np.ndarray) -> np.ndarray:
    """x = (y - mean) sqrt(n) / |y - mean| in FP32 (0 for a flat patch), as
    float64."""
    Y = np.asarray(Y, np.float32)
    n = Y.shape[1]
    C = (Y - Y.mean(axis=1, dtype=np.float64)[:, None].astype(np.float32)).astype(np.float32)
    ss = np.sum(C.astype(np.float64) ** 2, axis=1)
    sc = np.where(ss > 0, np.sqrt(n / np.where(ss > 0, ss, 1.0)), 0.0).astype(np.float32)
    return (C * sc[:, None]).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(params, Y, K: int, emulate: bool = True) -> dict:
    n = Y.shape[1]
    W1, b1, W2, b2, W3, b3 = unpack(params, n, K)
    r = bf16 if emulate else (lambda v: np.asarray(v, np.float64))
    X = r(inputs(Y))
    Z1 = X @ r(W1).T + b1
    H1 = r(gelu(Z1))
    Z2 = H1 @ r(W2).T + b2
    H2 = r(gelu(Z2))
    Z3 = H2 @ r(W3).T + b3
    return {"X": X, "Z1": Z1, "H1": H1, "Z2": Z2, "H2": H2, "Z3": Z3}


def target_mask(sup: np.ndarray, K: int) -> np.ndarray:
    sup = np.asarray(sup)
    T = np.zeros((sup.shape[0], K))
    rows, cols = np.nonzero(sup >= 0)
    T[rows, sup[rows, cols]] = 1.0
    return T


def loss_grad(params, Y, sup, K: int, emulate: bool = True):
    """(mean BCE loss, gradient in the parameter order) for the batch."""
    n = Y.shape[1]
    W1, b1, W2, b2, W3, b3 = unpack(params, n, K)
    r = bf16 if emulate else (lambda v: np.asarray(v, np.float64))
    f = forward(params, Y, K, emulate)
    B = Y.shape[0]
    T = target_mask(sup, K)
    Z3 = f["Z3"]
    loss = float(np.mean(np.maximum(Z3, 0) + np.log1p(np.exp(-np.abs(Z3))) - T * Z3))
    dZ3 = r((1.0 / (1.0 + np.exp(-Z3)) - T) / (B * K))
    dW3 = dZ3.T @ f["H2"]
    db3 = dZ3.sum(0)
    dZ2 = r((dZ3 @ r(W3)) * gelu_grad(f["Z2"]))
    dW2 = dZ2.T @ f["H1"]
    db2 = dZ2.sum(0)
    dZ1 = r((dZ2 @ r(W2)) * gelu_grad(f["Z1"]))
    dW1 = dZ1.T @ f["X"]
    db1 = dZ1.sum(0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return loss, g


def top_candidates(Z3: np.ndarray, C: int = 16) -> np.ndarray:
    """The C largest scores per row, best first, lower atom first on ties."""
    K = Z3.shape[1]
    order = np.lexsort((np.broadcast_to(np.arange(K), Z3.shape), -Z3), axis=1)
    return order[:, :C].astype(np.int32)


def omp_restricted(Y, D, cand, L: int):
    """The reference's pursuit (cublas_matrix_omp.cu:186-393) with the argmax
    over each patch's candidates only: -> (idx, coef, residual norms)."""
    Y = np.asarray(Y, np.float64)
    D = np.asarray(D, np.float64)
    G = D @ D.T
    N = Y.shape[0]
    idx = np.full((N, L), -1, np.int32)
    coef = np.zeros((N, L))
    rn = np.zeros(N)
    for p in range(N):
        y = Y[p]
        c = np.asarray(cand[p])
        b = D[c] @ y
        yy = float(y @ y)
        if yy == 0.0:
            idx[p, 0] = 0
            continue
        S = []
        g = np.zeros(0)
        rr = yy
        for step in range(L):
            if step > 0 and np.sqrt(max(rr, 0.0)) < 1e-3:
                break
            alpha = b - (G[np.ix_(c, S)] @ g if S else 0.0)
            key = np.abs(alpha)
            best = np.max(key)
            a = int(np.min(c[key == best]))
            if a in S:
                break
            S2 = S + [a]
            Gs = G[np.ix_(S2, S2)]
            try:
                Lc = np.linalg.cholesky(Gs)
            except np.linalg.LinAlgError:
                break
            bs = D[S2] @ y
            z = np.linalg.solve(Lc, bs)
            g = np.linalg.solve(Lc.T, z)
            S = S2
            rr = yy - float(z @ z)
        idx[p, :len(S)] = S
        coef[p, :len(S)] = g
        rn[p] = np.sqrt(max(rr, 0.0))
    return idx, coef, rn
