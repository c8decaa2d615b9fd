"""Host-side pieces of the implicit-adjoint check (CPU only): the perturbed
symmetric stencil, and the FP64 host adjoint built on the oracle's restatement
of CG_ref, pinned against a sparse direct solve and central finite differences."""
import numpy as np
import pytest

scipy = pytest.importorskip("scipy")
import scipy.sparse as sp  # noqa: E402
import scipy.sparse.linalg as spla  # noqa: E402

from hpcg_b200 import perturbed as PT  # noqa: E402


def sparse_from_slots(vals27, nx, ny, nz):
    n = nx * ny * nz
    i = np.arange(n)
    iz, rem = np.divmod(i, nx * ny)
    iy, ix = np.divmod(rem, nx)
    rows, cols, data = [], [], []
    for k in range(27):
        sx, sy, sz = k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1
        jx, jy, jz = ix + sx, iy + sy, iz + sz
        ok = (jx >= 0) & (jx < nx) & (jy >= 0) & (jy < ny) & (jz >= 0) & (jz < nz)
        rows.append(i[ok]); cols.append(((jz * ny + jy) * nx + jx)[ok]); data.append(vals27[ok, k])
    return sp.csr_matrix((np.concatenate(data), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))


def perturbed_levels(oracle, nx, ny, nz, vals27):
    """Oracle hierarchy: perturbed fine level, standard coarse levels."""
    P = oracle.generate(nx, ny, nz)
    nnz, cols, vals, diag = PT.to_reference_rows(vals27, nx, ny, nz)
    L0 = P.levels[0]
    P.levels[0] = oracle.Level(nx, ny, nz, nnz, cols, vals, diag, L0.f2c)
    return P.levels


def host_adjoint(oracle, levels, vals27, x, g, tol=1e-13):
    """FP64 host adjoint: lambda from the CG_ref restatement, dL/da_ij = -lambda_i x_j."""
    lam = oracle.cg(levels, g, np.zeros_like(g), 2000, tol)[0]
    nx, ny, nz = levels[0].nx, levels[0].ny, levels[0].nz
    n = nx * ny * nz
    i = np.arange(n)
    iz, rem = np.divmod(i, nx * ny)
    iy, ix = np.divmod(rem, nx)
    gv = np.zeros((n, 27))
    for k in range(27):
        sx, sy, sz = k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1
        jx, jy, jz = ix + sx, iy + sy, iz + sz
        ok = (jx >= 0) & (jx < nx) & (jy >= 0) & (jy < ny) & (jz >= 0) & (jz < nz)
        j = np.where(ok, (jz * ny + jy) * nx + jx, 0)
        gv[:, k] = np.where(ok, -lam * x[j], 0.0)
    return lam, gv


def central_difference_slot(v, b, xt, i, k, h, nx, ny, nz):
    """Central difference (L(a+h) - L(a-h)) / 2h of L = 0.5 ||x - xt||^2 for slot
    (i, k), evaluated without cancellation: with x- = A(a-h)^-1 b, the difference
    d = x+ - x- solves A(a+h) d = -2h e_i x-_j exactly, and
    L(a+h) - L(a-h) = 0.5 d'(2 x- + d - 2 xt)."""
    dv = np.zeros_like(v)
    dv[i, k] = h
    Am = sparse_from_slots(v - dv, nx, ny, nz).tocsc()
    Ap = sparse_from_slots(v + dv, nx, ny, nz).tocsc()
    xm = spla.spsolve(Am, b)
    sx, sy, sz = k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1
    iz, rem = divmod(i, nx * ny)
    iy, ix = divmod(rem, nx)
    j = ((iz + sz) * ny + (iy + sy)) * nx + (ix + sx)
    rhs = np.zeros_like(b)
    rhs[i] = -2.0 * h * xm[j]
    d = spla.spsolve(Ap, rhs)
    return 0.5 * np.dot(d, 2 * xm + d - 2 * xt) / (2 * h)


def central_difference_rhs(A, b, xt, x, i, h):
    """The same for b_i: d = x+ - x- = 2h A^-1 e_i, L+ - L- = d'(x - xt)."""
    e = np.zeros_like(b)
    e[i] = 2.0 * h
    d = spla.spsolve(A, e)
    return np.dot(d, x - xt) / (2 * h)


def test_perturbed_stencil_is_symmetric_and_dominant():
    nx = ny = nz = 8
    v = PT.perturbed_values(nx, ny, nz)
    A = sparse_from_slots(v, nx, ny, nz)
    assert abs(A - A.T).max() == 0.0
    off = np.abs(np.delete(v, 13, axis=1)).sum(1)
    assert np.allclose(v[:, 13], 1.05 * off)
    offv = np.delete(v, 13, axis=1)
    offv = offv[offv != 0]
    assert np.all(offv <= -0.9) and np.all(offv >= -1.1)
    assert np.array_equal(v, PT.perturbed_values(nx, ny, nz))  # seeded


def test_reference_rows_match_slots(oracle):
    nx, ny, nz = 8, 6, 4
    v = PT.perturbed_values(nx, ny, nz)
    nnz, cols, vals, diag = PT.to_reference_rows(v, nx, ny, nz)
    L = oracle.Level(nx, ny, nz, nnz, cols, vals, diag)
    x = np.random.default_rng(0).standard_normal(nx * ny * nz)
    assert np.allclose(oracle.spmv(L, x), sparse_from_slots(v, nx, ny, nz) @ x, rtol=1e-14, atol=1e-13)


def test_host_adjoint_against_direct_solve_and_fd(oracle):
    nx = ny = nz = 8
    n = nx * ny * nz
    v = PT.perturbed_values(nx, ny, nz)
    b = PT.rhs_uniform(n)
    xt = PT.target_normal(n)
    levels = perturbed_levels(oracle, nx, ny, nz, v)
    A = sparse_from_slots(v, nx, ny, nz).tocsc()
    x = spla.spsolve(A, b)
    xo = oracle.cg(levels, b, np.zeros(n), 2000, 1e-13)[0]
    assert np.max(np.abs(xo - x)) <= 1e-10 * np.max(np.abs(x))
    g = x - xt
    lam, gv = host_adjoint(oracle, levels, v, x, g)
    assert np.max(np.abs(lam - spla.spsolve(A.T, g))) <= 1e-10 * np.max(np.abs(lam))
    rng = np.random.default_rng(7)
    h = 1e-6
    checked = 0
    while checked < 8:
        i, k = int(rng.integers(n)), int(rng.integers(27))
        if v[i, k] == 0.0:
            continue
        fd = central_difference_slot(v, b, xt, i, k, h, nx, ny, nz)
        assert abs(fd - gv[i, k]) <= 1e-6 * abs(gv[i, k]), (i, k, fd, gv[i, k])
        checked += 1
    for i in rng.integers(n, size=4):
        fd = central_difference_rhs(A, b, xt, x, int(i), h)
        assert abs(fd - lam[i]) <= 1e-6 * abs(lam[i])
