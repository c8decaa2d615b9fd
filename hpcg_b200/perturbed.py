"""The perturbed symmetric 27-point stencil used to check the implicit adjoint.

Off-diagonal a_ij = a_ji = -(1 + 0.1 u_ij) with u_ij ~ U[-1, 1) drawn from a
seeded hash of the unordered pair {i, j} (so A is symmetric by construction);
diagonal a_ii = 1.05 * sum_j |a_ij| (strictly diagonally dominant). Only the
fine level is perturbed: the coarse levels stay the standard stencil, as
GenerateCoarseProblem.cpp:97 regenerates them.

Values are returned in the library's direction-slot form: float64 [n, 27],
rows in natural order, value k of row i belonging to stencil direction
k = (sz+1)*9 + (sy+1)*3 + (sx+1) (0 where the direction leaves the grid), which
is what hpcg_b200_set_values takes.
"""
from __future__ import annotations

import numpy as np

SEED = 0x48504347
_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(z: np.ndarray) -> np.ndarray:
    """The splitmix64 finaliser (Steele, Lea, Flood 2014) on uint64 arrays."""
    z = z.astype(np.uint64)
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def pair_uniform(i: np.ndarray, j: np.ndarray, n: int, seed: int = SEED) -> np.ndarray:
    """u in [-1, 1) for the unordered pairs (i, j) of an n-row grid."""
    lo = np.minimum(i, j).astype(np.uint64)
    hi = np.maximum(i, j).astype(np.uint64)
    with np.errstate(over="ignore"):
        key = lo * np.uint64(n) + hi
    h = splitmix64(key ^ splitmix64(np.full(key.shape, seed, dtype=np.uint64)))
    return (h >> np.uint64(11)).astype(np.float64) * (2.0 ** -53) * 2.0 - 1.0


def perturbed_values(nx: int, ny: int, nz: int, seed: int = SEED) -> np.ndarray:
    n = nx * ny * nz
    i = np.arange(n, dtype=np.int64)
    iz, rem = np.divmod(i, nx * ny)
    iy, ix = np.divmod(rem, nx)
    vals = np.zeros((n, 27))
    absum = np.zeros(n)
    for k in range(27):
        if k == 13:
            continue
        sx, sy, sz = k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1
        jx, jy, jz = ix + sx, iy + sy, iz + sz
        ok = (jx >= 0) & (jx < nx) & (jy >= 0) & (jy < ny) & (jz >= 0) & (jz < nz)
        j = (jz * ny + jy) * nx + jx
        a = -(1.0 + 0.1 * pair_uniform(i, j, n, seed))
        a = np.where(ok, a, 0.0)
        vals[:, k] = a
        absum += np.abs(a)
    vals[:, 13] = 1.05 * absum
    return vals


def rhs_uniform(n: int, seed: int = SEED) -> np.ndarray:
    """b ~ U[-1, 1] (numpy PCG64 from `seed`)."""
    return np.random.Generator(np.random.PCG64(seed)).uniform(-1.0, 1.0, n)


def target_normal(n: int, seed: int = SEED + 1) -> np.ndarray:
    """x_target ~ N(0, 1) (numpy PCG64 from `seed`)."""
    return np.random.Generator(np.random.PCG64(seed)).standard_normal(n)


def to_reference_rows(vals27: np.ndarray, nx: int, ny: int, nz: int):
    """The same matrix in the reference's row layout: (nnz, cols, vals) with up to
    27 entries per row in entry order (lexicographic directions, out-of-grid
    directions dropped), padded to 27 with column i and value 0."""
    n = nx * ny * nz
    i = np.arange(n, dtype=np.int64)
    iz, rem = np.divmod(i, nx * ny)
    iy, ix = np.divmod(rem, nx)
    cols = np.repeat(i[:, None], 27, axis=1).astype(np.int32)
    out = np.zeros((n, 27))
    nnz = np.zeros(n, np.int32)
    diag = np.zeros(n, np.int32)
    for k in range(27):
        sx, sy, sz = k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1
        jx, jy, jz = ix + sx, iy + sy, iz + sz
        ok = (jx >= 0) & (jx < nx) & (jy >= 0) & (jy < ny) & (jz >= 0) & (jz < nz)
        j = (jz * ny + jy) * nx + jx
        rows = np.nonzero(ok)[0]
        slot = nnz[rows]
        cols[rows, slot] = j[rows]
        out[rows, slot] = vals27[rows, k]
        if k == 13:
            diag[rows] = slot
        nnz[rows] += 1
    return nnz, cols.reshape(-1), out.reshape(-1), diag
