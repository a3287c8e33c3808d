"""CPU restatement of the serving engine's three request kinds (numpy).

TEST INFRASTRUCTURE ONLY: used by tests/ to check the engine
(ops_b200/csrc/serve/ob2_serve.cu); nothing in the product imports it.

  * 2D Poisson: right-hand side b = h^2 (2 U - 1) from the counter-based hash,
    h = 1 / (n + 1), and the 5-point operator A x = 4 x - (neighbours) with a
    zero Dirichlet boundary; `relative_residual` measures ||b - A x|| / ||b||,
    the engine's stopping quantity, for a solution computed on the GPU.
  * 2D implicit heat: u0 = 2 U - 1 from the hash (stream 3), each step solves
    (1 + 4 rho) u' - rho (neighbours of u') = u with rho = dt / h^2 = 1 and a
    zero Dirichlet boundary; `heat_steps` solves the same steps with a
    direct sparse solver, `heat_relative_residual` measures one step.
  * 3D ADI heat step, after the reference's adi app: the right-hand side of
    apps/c/adi/preproc_kernel.h (d = lambda * (sum of the six neighbours -
    6 u) inside, 0 on the Dirichlet boundary; a = c = -lambda/2, b = 1 +
    lambda inside, identity rows on the boundary), then the Thomas algorithm
    along x and y on d and along z with the solution added to u (the
    ops_tridMultiDimBatch / _Inc calls of apps/c/adi/adi.cpp:406-420).  The
    forward sweep multiplies by the precomputed 1/(b_i - a_i c'_{i-1}), as
    the engine does, so the arithmetic is the same operation for operation.
    Deviation from the reference's adi app, stated: the serving engine's ADI
    requests have constant coefficients, so it precomputes the Thomas
    coefficients c'_i and 1 / (b_i - a_i c'_{i-1}) once per size and stores only
    u and the right-hand side (72 B per point per step instead of the 216 B of
    the adi app's per-point a, b, c arrays, which the ADI configuration of
    apps/adi3d keeps); the solution is the same up to round-off.
"""

from __future__ import annotations

import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def hash_uniform(seed: int, i, j, k):
    """U[0,1) from the splitmix64 finaliser of (seed, i, j, k); i, j, k arrays."""
    with np.errstate(over="ignore"):
        z = ((np.uint64(seed) << np.uint64(42)) ^ (np.asarray(i, np.uint64) << np.uint64(21)) ^
             np.asarray(j, np.uint64) ^ (np.asarray(k, np.uint64) << np.uint64(52)))
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def poisson_rhs(n: int, seed: int) -> np.ndarray:
    """b[j, i] (row j = y) of an n x n request."""
    j, i = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    h = 1.0 / (n + 1)
    return h * h * (2.0 * hash_uniform(seed, i, j, 0) - 1.0)


def poisson_apply(x: np.ndarray) -> np.ndarray:
    p = np.zeros((x.shape[0] + 2, x.shape[1] + 2))
    p[1:-1, 1:-1] = x
    return (4.0 * p[1:-1, 1:-1] - p[1:-1, :-2] - p[1:-1, 2:] - p[:-2, 1:-1] - p[2:, 1:-1])


def relative_residual(x: np.ndarray, seed: int) -> float:
    n = x.shape[0]
    b = poisson_rhs(n, seed)
    return float(np.linalg.norm(b - poisson_apply(x)) / np.linalg.norm(b))


def adi_init(n: int, seed: int) -> np.ndarray:
    """u[z, y, x]"""
    z, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    return 2.0 * hash_uniform(seed, i, j, z + 1) - 1.0


def thomas_coefs(n: int, lam: float):
    a, b, c = -0.5 * lam, 1.0 + lam, -0.5 * lam
    cp = np.zeros(n)
    mm = np.zeros(n)
    mm[0] = 1.0
    for i in range(1, n):
        edge = i == n - 1
        ai, bi, ci = (0.0, 1.0, 0.0) if edge else (a, b, c)
        mm[i] = 1.0 / (bi - ai * cp[i - 1])
        cp[i] = ci * mm[i]
    arow = np.full(n, a)
    arow[0] = 0.0
    arow[n - 1] = 0.0
    return arow, cp, mm


def thomas_along(d: np.ndarray, axis: int, lam: float) -> np.ndarray:
    """solution of the constant-coefficient system along `axis` of d"""
    n = d.shape[axis]
    arow, cp, mm = thomas_coefs(n, lam)
    v = np.moveaxis(d.copy(), axis, 0)
    v[0] = v[0] * mm[0]
    for m in range(1, n):
        v[m] = (v[m] - arow[m] * v[m - 1]) * mm[m]
    for m in range(n - 2, -1, -1):
        v[m] = v[m] - cp[m] * v[m + 1]
    return np.moveaxis(v, 0, axis)


def adi_steps(n: int, seed: int, steps: int, lam: float = 1.0) -> np.ndarray:
    u = adi_init(n, seed)
    for _ in range(steps):
        d = np.zeros_like(u)
        c = u[1:-1, 1:-1, 1:-1]
        s = (u[1:-1, 1:-1, :-2] + u[1:-1, 1:-1, 2:] + u[1:-1, :-2, 1:-1] + u[1:-1, 2:, 1:-1] +
             u[:-2, 1:-1, 1:-1] + u[2:, 1:-1, 1:-1])
        d[1:-1, 1:-1, 1:-1] = lam * (s - 6.0 * c)
        d = thomas_along(d, 2, lam)  # x
        d = thomas_along(d, 1, lam)  # y
        u = u + thomas_along(d, 0, lam)  # z, added to u
    return u


HEAT_RHO = 1.0


def heat_init(n: int, seed: int) -> np.ndarray:
    """u0[j, i] of an n x n heat request."""
    j, i = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    return 2.0 * hash_uniform(seed, i, j, 3) - 1.0


def heat_apply(x: np.ndarray, rho: float = HEAT_RHO) -> np.ndarray:
    p = np.zeros((x.shape[0] + 2, x.shape[1] + 2))
    p[1:-1, 1:-1] = x
    return (1.0 + 4.0 * rho) * p[1:-1, 1:-1] - rho * (p[1:-1, :-2] + p[1:-1, 2:] + p[:-2, 1:-1] +
                                                      p[2:, 1:-1])


def heat_relative_residual(x: np.ndarray, b: np.ndarray) -> float:
    return float(np.linalg.norm(b - heat_apply(x)) / np.linalg.norm(b))


def heat_steps(n: int, seed: int, steps: int, rho: float = HEAT_RHO) -> np.ndarray:
    """the exact implicit steps (sparse direct solve) from heat_init"""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    e = np.ones(n)
    t = sp.diags([-rho * e[:-1], -rho * e[:-1]], [-1, 1])
    eye = sp.identity(n)
    a = (sp.kron(eye, t) + sp.kron(t, eye) + (1.0 + 4.0 * rho) * sp.identity(n * n)).tocsc()
    u = heat_init(n, seed).reshape(-1)
    lu = spla.splu(a)
    for _ in range(steps):
        u = lu.solve(u)
    return u.reshape(n, n)
