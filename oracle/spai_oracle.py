"""CPU oracle of the learned SPAI preconditioner (TEST INFRASTRUCTURE ONLY).

The learned sparse approximate inverse has no counterpart in the reference
MCLS, so this module restates the library's own definition of it in numpy:
features, the 16-64-64-16 ReLU network, the values of M on A's pattern, the
training loss (1/R) sum_v |v - M A v|^2 / |v|^2 and its gradient through the
network.  Two flavours:

* ``rounded=True`` mirrors the device arithmetic: BF16 operands (round to
  nearest even) at the points where the tensor-core kernels round, products
  accumulated exactly and rounded to FP32 at the accumulator;
* ``rounded=False`` is plain FP64 with no rounding, whose analytic gradient
  the tests pin against central finite differences of the loss.

Only the tests and ``__graft_entry__.smoke()`` import this module.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

F, H, O = 16, 64, 16
W1, B1 = 0, H * F
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + O * H
NPARAMS = B3 + O


def bf16(x):
    """Round FP32 values to BF16 (nearest, ties to even), returned as FP32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(x.shape)


def unpack(p):
    p = np.asarray(p)
    if p.dtype != np.float64:
        p = p.astype(np.float32)
    return (p[W1:B1].reshape(H, F), p[B1:W2], p[W2:B2].reshape(H, H), p[B2:W3],
            p[W3:B3].reshape(O, H), p[B3:NPARAMS])


def stencil(A):
    """Sorted distinct column offsets of A and its diagonal-offset values
    dia[s, i] = A[i, i + off[s]] (0 where absent)."""
    A = sp.csr_matrix(A)
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    d = A.indices - rows
    offs = np.unique(d)
    dia = np.zeros((len(offs), A.shape[0]))
    s = np.searchsorted(offs, d)
    dia[s, rows] = A.data
    return offs, dia


def features(A):
    """[n, 16] features of every row (FP32, before BF16 rounding)."""
    offs, dia = stencil(A)
    n = dia.shape[1]
    c = int(np.where(offs == 0)[0][0])
    aii = dia[c]
    X = np.zeros((n, F), dtype=np.float32)
    q = 0
    i = np.arange(n)
    for s, o in enumerate(offs):
        if o == 0:
            continue
        a = dia[s]
        j = i + o
        ok = (a != 0.0) & (j >= 0) & (j < n)
        jj = np.clip(j, 0, n - 1)
        X[:, 2 * q] = np.where(ok, a / aii, 0.0).astype(np.float32)
        X[:, 2 * q + 1] = np.where(ok, np.log(np.where(ok, dia[c][jj] / aii, 1.0)), 0.0).astype(
            np.float32)
        q += 1
    return X


def _mm(a, b, rounded):
    r = a.astype(np.float64) @ b.astype(np.float64)
    return r.astype(np.float32) if rounded else r


def forward(params, X, rounded=True):
    """Network outputs [n, 16] and the activations the backward pass needs."""
    w1, b1, w2, b2, w3, b3 = unpack(params)
    R = bf16 if rounded else (lambda v: np.asarray(v, dtype=np.float64))
    Xr = R(X)
    Z1 = _mm(Xr, R(w1).T, rounded) + b1
    H1 = R(np.maximum(Z1, 0))
    Z2 = _mm(H1, R(w2).T, rounded) + b2
    H2 = R(np.maximum(Z2, 0))
    out = _mm(H2, R(w3).T, rounded) + b3
    return out, (Xr, H1, H2)


def mvalues(A, out):
    """Values of M on A's CSR pattern: (delta + out_s) / A_ii."""
    A = sp.csr_matrix(A)
    offs, dia = stencil(A)
    c = int(np.where(offs == 0)[0][0])
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    d = A.indices - rows
    s = np.searchsorted(offs, d)
    o = np.asarray(out, dtype=np.float64)[rows, s]
    return ((d == 0).astype(np.float64) + o) / dia[c][rows]


def loss_grad(A, mvals, V, pen_w=0.0, pen_c=1.0):
    """Loss and dL/dout [n, 16] for vectors V [R, n] (FP64).  pen_w > 0 adds
    pen_w/n * sum_i max(0, W_i - pen_c)^2, W_i = sum_j |(I - M A)_ij|."""
    A = sp.csr_matrix(A)
    n = A.shape[0]
    offs, dia = stencil(A)
    c = int(np.where(offs == 0)[0][0])
    M = sp.csr_matrix((mvals, A.indices, A.indptr), shape=A.shape)
    rows = np.repeat(np.arange(n), np.diff(A.indptr))
    s = np.searchsorted(offs, A.indices - rows)
    G = np.zeros((n, O))
    loss = 0.0
    R = V.shape[0]
    for v in V:
        w = 1.0 / (R * float(v @ v))
        z = A @ v
        e = v - M @ z
        loss += w * float(e @ e)
        contrib = -2.0 * w * e[rows] * z[A.indices] / dia[c][rows]
        np.add.at(G, (rows, s), contrib)
    if pen_w > 0.0:
        H = (sp.identity(n) - M @ A).tocsr()
        H.sum_duplicates()
        W = np.asarray(abs(H).sum(1)).ravel()
        pen = np.maximum(W - pen_c, 0.0)
        loss += pen_w * float(pen @ pen) / n
        # dW_i/dM_ik = -sum_j sign(H_ij) A_kj over the entries (i, k) of M.
        S = H.copy()
        S.data = np.sign(S.data)
        dW = -(S @ A.T).tocsr()  # dW[i, k]
        coef = 2.0 * pen_w * pen / n
        dWik = np.asarray(dW[rows, A.indices]).ravel()
        np.add.at(G, (rows, s), coef[rows] * dWik / dia[c][rows])
    return loss, G


def backward(params, acts, G, rounded=True):
    """Parameter gradient (flat, FP64) from dL/dout."""
    w1, b1, w2, b2, w3, b3 = unpack(params)
    Xr, H1, H2 = acts
    R = bf16 if rounded else (lambda v: np.asarray(v, dtype=np.float64))
    Gr = R(np.asarray(G, dtype=np.float32) if rounded else G)
    dH2 = _mm(Gr, R(w3), rounded)
    dZ2 = R(np.where(H2 > 0, dH2, 0))
    dH1 = _mm(dZ2, R(w2), rounded)
    dZ1 = R(np.where(H1 > 0, dH1, 0))
    g = np.zeros(NPARAMS)
    f64 = lambda a: np.asarray(a, dtype=np.float64)
    g[W3:B3] = (f64(Gr).T @ f64(H2)).ravel()
    g[B3:NPARAMS] = f64(Gr).sum(0)
    g[W2:B2] = (f64(dZ2).T @ f64(H1)).ravel()
    g[B2:W3] = f64(dZ2).sum(0)
    g[W1:B1] = (f64(dZ1).T @ f64(Xr)).ravel()
    g[B1:W2] = f64(dZ1).sum(0)
    return g


def loss_and_gradient(params, A, V, rounded=True, pen_w=0.0, pen_c=1.0):
    """Loss and parameter gradient of the whole chain on (A, V)."""
    X = features(A)
    out, acts = forward(params, X, rounded)
    m = mvalues(A, out)
    loss, G = loss_grad(A, m, V, pen_w, pen_c)
    return loss, backward(params, acts, G, rounded)


def init_params(seed, zero_last=True):
    """He-uniform hidden layers; the output layer zero (Jacobi) or small."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAMS, dtype=np.float32)
    p[W1:B1] = np.sqrt(6.0 / F) * rng.uniform(-1, 1, H * F)
    p[W2:B2] = np.sqrt(6.0 / H) * rng.uniform(-1, 1, H * H)
    if not zero_last:
        p[B1:W2] = 0.1 * rng.uniform(-1, 1, H)
        p[B2:W3] = 0.1 * rng.uniform(-1, 1, H)
        p[W3:B3] = 0.05 * rng.uniform(-1, 1, O * H)
        p[B3:NPARAMS] = 0.05 * rng.uniform(-1, 1, O)
    return p


def rho(A, mvals, iters=400, seed=0):
    """Power-iteration estimate of rho(I - M A)."""
    A = sp.csr_matrix(A)
    M = sp.csr_matrix((mvals, A.indices, A.indptr), shape=A.shape)
    v = np.random.default_rng(seed).uniform(-1, 1, A.shape[0])
    v /= np.linalg.norm(v)
    g = []
    for _ in range(iters):
        w = v - M @ (A @ v)
        nv = np.linalg.norm(w)
        g.append(nv)
        v = w / nv
    return float(np.exp(np.mean(np.log(g[-10:]))))
