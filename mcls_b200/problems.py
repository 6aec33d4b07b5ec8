"""Seeded synthetic linear systems for the MCSA workloads.

Every generator returns a ``scipy.sparse.csr_matrix`` (FP64, sorted column
indices) and, where the workload defines one, a right-hand side.  The
discretisations follow the workload definitions:

* 2D Poisson, 5-point finite differences on an ``nx x ny`` interior grid with
  Dirichlet zero boundaries eliminated (``h = 1/(nx+1)``).
* 3D variable-coefficient diffusion, 7-point finite volumes on an ``n^3``
  grid: per-cell coefficient, harmonic-mean face coefficients, boundary faces
  use the cell value against a Dirichlet zero boundary, plus absorption.
* 3D diffusion-reaction with piecewise-constant coefficients on material
  blocks.
* 2D anisotropic diffusion with a rotated diffusion tensor on a 9-point
  stencil (mixed-sign off-diagonals).
* The tridiagonal (1, -0.14) system of the reference's MCSA tests.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _csr(A):
    A = sp.csr_matrix(A)
    A.sum_duplicates()
    A.sort_indices()
    A.eliminate_zeros()
    return A


def tridiag_test(n: int = 10, diag: float = 1.0, off: float = -0.14):
    """Tridiagonal system of tpetra/test/tstTpetraMCSASolverManager.cpp:91-116.

    The first and last rows carry an explicit 0.0 entry (three entries each),
    as the reference inserts them; Tpetra keeps explicit zeros.
    """
    rows, cols, vals = [], [], []
    for i in range(n):
        if i == 0:
            cs, vs = [0, 1, 2], [diag, off, 0.0]
        elif i == n - 1:
            cs, vs = [n - 3, n - 2, n - 1], [0.0, off, diag]
        else:
            cs, vs = [i - 1, i, i + 1], [off, diag, off]
        rows += [i] * 3
        cols += cs
        vals += vs
    A = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    A.sort_indices()
    return A


def fixed_point_test(n: int = 10):
    """System of tpetra/test/tstTpetraFixedPointSolverManager.cpp:89-116:
    interior rows 0.14 / 1 / 0.14; the first row holds 0.14, 0.14, 1 at
    columns 0, 1, 2 and the last row 0.14, 0.14, 1 at n-3, n-2, n-1."""
    rows, cols, vals = [], [], []
    for i in range(n):
        if i == 0:
            cs, vs = [0, 1, 2], [0.14, 0.14, 1.0]
        elif i == n - 1:
            cs, vs = [n - 3, n - 2, n - 1], [0.14, 0.14, 1.0]
        else:
            cs, vs = [i - 1, i, i + 1], [0.14, 1.0, 0.14]
        rows += [i] * 3
        cols += cs
        vals += vs
    A = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    A.sort_indices()
    return A


def poisson2d(nx: int, ny: int | None = None):
    """5-point Laplacian, A_ii = 4/h^2, A_ij = -1/h^2, h = 1/(nx+1)."""
    ny = nx if ny is None else ny
    h = 1.0 / (nx + 1)
    inv = 1.0 / (h * h)
    N = nx * ny
    i = np.arange(N)
    x = i % nx
    main = np.full(N, 4.0 * inv)
    east = np.where(x[:-1] < nx - 1, -inv, 0.0)
    north = np.full(N - nx, -inv)
    A = sp.diags([main, east, east, north, north], [0, 1, -1, nx, -nx],
                 shape=(N, N), format="csr")
    return _csr(A)


def _diffusion3d(D: np.ndarray, sigma: np.ndarray, h: float):
    """7-point finite-volume operator for per-cell D and sigma (shape n^3)."""
    n = D.shape[0]
    N = n ** 3
    inv = 1.0 / (h * h)
    Dflat = D.reshape(N)

    def face(a, b):
        return 2.0 * a * b / (a + b)

    diag = sigma.reshape(N).astype(np.float64).copy()
    offs = []
    vals = []
    # axis order: index = x + n*y + n*n*z  (x fastest)
    for axis, stride in ((2, 1), (1, n), (0, n * n)):
        Df = face(np.take(D, range(0, n - 1), axis=axis), np.take(D, range(1, n), axis=axis))
        # face between cell c and c+stride along axis
        full = np.zeros_like(D)
        sl = [slice(None)] * 3
        sl[axis] = slice(0, n - 1)
        full[tuple(sl)] = Df
        up = full.reshape(N)  # coefficient to the + neighbour
        full2 = np.zeros_like(D)
        sl2 = [slice(None)] * 3
        sl2[axis] = slice(1, n)
        full2[tuple(sl2)] = Df
        dn = full2.reshape(N)  # coefficient to the - neighbour
        # boundary faces (Dirichlet zero): cell coefficient
        lo = [slice(None)] * 3
        lo[axis] = 0
        hi = [slice(None)] * 3
        hi[axis] = n - 1
        bnd = np.zeros_like(D)
        bnd[tuple(lo)] += D[tuple(lo)]
        bnd[tuple(hi)] += D[tuple(hi)]
        diag += (up + dn + bnd.reshape(N)) * inv
        offs += [stride, -stride]
        vals += [-up[: N - stride] * inv, -dn[stride:] * inv]
    A = sp.diags([diag] + vals, [0] + offs, shape=(N, N), format="csr")
    return _csr(A)


def diffusion3d_varcoef(n: int = 128, seed: int = 0, sigma_a: float = 0.01,
                        dmin: float = 0.1, dmax: float = 10.0):
    """3D 7-point variable-coefficient diffusion, D log-uniform per cell."""
    rng = np.random.Generator(np.random.PCG64(seed))
    D = np.exp(rng.uniform(np.log(dmin), np.log(dmax), size=(n, n, n)))
    h = 1.0 / (n + 1)
    A = _diffusion3d(D, np.full((n, n, n), sigma_a), h)
    b = rng.uniform(0.0, 1.0, size=n ** 3)
    return A, b


def diffusion3d_blocks(n: int = 256, blocks: int = 8, seed: int = 0):
    """3D diffusion-reaction, piecewise-constant (D, sigma_a) on blocks^3."""
    rng = np.random.Generator(np.random.PCG64(seed))
    Db = rng.uniform(0.5, 5.0, size=(blocks,) * 3)
    Sb = rng.uniform(0.001, 0.1, size=(blocks,) * 3)
    rep = n // blocks
    D = np.repeat(np.repeat(np.repeat(Db, rep, 0), rep, 1), rep, 2)
    S = np.repeat(np.repeat(np.repeat(Sb, rep, 0), rep, 1), rep, 2)
    h = 1.0 / (n + 1)
    A = _diffusion3d(D, S, h)
    b = rng.uniform(0.0, 1.0, size=n ** 3)
    return A, b


def anisotropic2d(n: int, ratio: float, theta: float):
    """9-point FD stencil of -div(K grad u), K = R diag(1, 1/ratio) R^T."""
    c, s = np.cos(theta), np.sin(theta)
    k1, k2 = 1.0, 1.0 / ratio
    kxx = k1 * c * c + k2 * s * s
    kyy = k1 * s * s + k2 * c * c
    kxy = (k1 - k2) * c * s
    h = 1.0 / (n + 1)
    inv = 1.0 / (h * h)
    N = n * n
    i = np.arange(N)
    x = i % n
    y = i // n
    main = np.full(N, (2 * kxx + 2 * kyy) * inv)
    offs = [0]
    vals = [main]
    stencil = {
        (1, 0): -kxx * inv, (-1, 0): -kxx * inv,
        (0, 1): -kyy * inv, (0, -1): -kyy * inv,
        (1, 1): -0.5 * kxy * inv, (-1, -1): -0.5 * kxy * inv,
        (1, -1): 0.5 * kxy * inv, (-1, 1): 0.5 * kxy * inv,
    }
    for (dx, dy), v in stencil.items():
        off = dx + n * dy
        valid = (x + dx >= 0) & (x + dx < n) & (y + dy >= 0) & (y + dy < n)
        d = np.where(valid, v, 0.0)
        if off >= 0:
            vals.append(d[: N - off])
        else:
            vals.append(d[-off:])
        offs.append(off)
    A = sp.diags(vals, offs, shape=(N, N), format="csr")
    return _csr(A)


def anisotropic2d_sample(n: int, seed: int):
    """One seeded anisotropic system: ratio log-uniform [1,100], angle U[0,pi)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ratio = float(np.exp(rng.uniform(0.0, np.log(100.0))))
    theta = float(rng.uniform(0.0, np.pi))
    A = anisotropic2d(n, ratio, theta)
    b = rng.uniform(0.0, 1.0, size=n * n)
    return A, b, ratio, theta


def _diffusion2d(D: np.ndarray, sigma: np.ndarray, h: float):
    """5-point finite-volume operator for per-cell D and sigma (shape n x n),
    harmonic face coefficients, Dirichlet zero boundary (cell coefficient)."""
    n = D.shape[0]
    N = n * n
    inv = 1.0 / (h * h)
    diag = sigma.reshape(N).astype(np.float64).copy()
    offs, vals = [], []
    for axis, stride in ((1, 1), (0, n)):
        a = np.take(D, range(0, n - 1), axis=axis)
        b = np.take(D, range(1, n), axis=axis)
        Df = 2.0 * a * b / (a + b)
        up = np.zeros_like(D)
        dn = np.zeros_like(D)
        sl = [slice(None)] * 2
        sl[axis] = slice(0, n - 1)
        up[tuple(sl)] = Df
        sl[axis] = slice(1, n)
        dn[tuple(sl)] = Df
        bnd = np.zeros_like(D)
        lo = [slice(None)] * 2
        hi = [slice(None)] * 2
        lo[axis] = 0
        hi[axis] = n - 1
        bnd[tuple(lo)] += D[tuple(lo)]
        bnd[tuple(hi)] += D[tuple(hi)]
        diag += (up.reshape(N) + dn.reshape(N) + bnd.reshape(N)) * inv
        offs += [stride, -stride]
        vals += [-up.reshape(N)[: N - stride] * inv, -dn.reshape(N)[stride:] * inv]
    A = sp.diags([diag] + vals, [0] + offs, shape=(N, N), format="csr")
    return _csr(A)


def batch_sample(count: int, nmin: float, nmax: float, seed: int = 0, rhs_max: int = 16):
    """Batched workload: `count` systems, each 2D Poisson / 2D var-coef / 3D
    Poisson / 3D var-coef with probability 1/4, N log-uniform in
    [nmin, nmax] rounded to the nearest square or cube grid, 1..rhs_max
    right-hand sides uniform(0, 1) each (coefficients log-uniform in
    [0.1, 10] per cell, absorption 0.01 for the var-coef kinds)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    systems, nrhs, rhs, kinds = [], [], [], []
    for _ in range(count):
        kind = int(rng.integers(0, 4))
        N = float(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        if kind < 2:
            n = max(3, int(round(np.sqrt(N))))
            if kind == 0:
                A = poisson2d(n)
            else:
                D = np.exp(rng.uniform(np.log(0.1), np.log(10.0), size=(n, n)))
                A = _diffusion2d(D, np.full((n, n), 0.01), 1.0 / (n + 1))
        else:
            n = max(3, int(round(N ** (1.0 / 3.0))))
            if kind == 2:
                A = _diffusion3d(np.ones((n, n, n)), np.zeros((n, n, n)), 1.0 / (n + 1))
            else:
                D = np.exp(rng.uniform(np.log(0.1), np.log(10.0), size=(n, n, n)))
                A = _diffusion3d(D, np.full((n, n, n), 0.01), 1.0 / (n + 1))
        r = int(rng.integers(1, rhs_max + 1))
        systems.append(A)
        nrhs.append(r)
        rhs.append(rng.uniform(0.0, 1.0, size=(A.shape[0], r)))
        kinds.append(("poisson2d", "varcoef2d", "poisson3d", "varcoef3d")[kind])
    return systems, nrhs, rhs, kinds
