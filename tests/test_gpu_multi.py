"""Several right-hand sides at once (hpcg_b200_cg_multi / _mg_multi): each
system's V-cycle is bitwise the single-system hpcg_b200_mg, and the lockstep CG
follows each system's single-system CG (same tolerances as the other CG tests:
|ours - single| <= 1e-10 * max(single, 1e-9) on the scaled residual)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def prob(binding):
    P = binding.Problem.generate(32)
    yield P
    P.free()


@pytest.mark.parametrize("nrhs", [1, 3, 8])
def test_mg_multi_is_single_mg_bitwise(prob, nrhs):
    n = prob.nrow
    r = np.random.default_rng(nrhs).standard_normal((nrhs, n))
    z = np.zeros((nrhs, n))
    prob.ComputeMG_multi(r, z)
    for j in range(nrhs):
        zj = np.zeros(n)
        prob.ComputeMG(np.ascontiguousarray(r[j]), zj)
        assert np.array_equal(z[j], zj), j


def test_cg_multi_follows_single_solves(prob):
    n = prob.nrow
    rng = np.random.Generator(np.random.PCG64(0x48504347))
    b = rng.uniform(-1.0, 1.0, (8, n))
    b[0] = prob.get_rhs()
    for max_iter in (1, 7, 25):
        x = np.zeros((8, n))
        ni, nr, nr0 = prob.CG_multi(b, x, max_iter, 0.0)
        for j in range(8):
            xs = np.zeros(n)
            ni_s, nr_s, nr0_s = prob.CG(np.ascontiguousarray(b[j]), xs, max_iter, 0.0, True)
            assert ni[j] == ni_s == max_iter
            assert abs(nr0[j] - nr0_s) <= 1e-13 * nr0_s
            s = nr_s / nr0_s
            assert abs(nr[j] / nr0[j] - s) <= 1e-10 * max(s, 1e-9), (j, nr[j] / nr0[j], s)
            assert np.max(np.abs(x[j] - xs)) <= 1e-9 * max(np.max(np.abs(xs)), 1.0)


def test_cg_multi_tolerance_per_system(prob):
    n = prob.nrow
    rng = np.random.Generator(np.random.PCG64(7))
    b = rng.uniform(-1.0, 1.0, (4, n))
    b[2] *= 1e-3  # same relative tolerance, different scale
    x = np.zeros((4, n))
    ni, nr, nr0 = prob.CG_multi(b, x, 500, 1e-9)
    for j in range(4):
        assert nr[j] / nr0[j] <= 1e-9
        xs = np.zeros(n)
        ni_s, nr_s, nr0_s = prob.CG(np.ascontiguousarray(b[j]), xs, 500, 1e-9, True)
        assert abs(int(ni[j]) - ni_s) <= 1
        assert np.linalg.norm(x[j] - xs) <= 1e-7 * np.linalg.norm(xs)


def test_cg_multi_zero_rhs_and_device_vectors(prob):
    import torch
    n = prob.nrow
    b = torch.zeros((2, n), dtype=torch.float64, device="cuda")
    b[1] = torch.from_numpy(prob.get_rhs()).cuda()
    x = torch.zeros_like(b)
    ni, nr, nr0 = prob.CG_multi(b, x, 50, 1e-8)
    assert ni[0] == 0 and nr0[0] == 0.0          # 0/0 > tol is false: no iterations, as CG.cpp:100
    assert torch.all(x[0] == 0)
    assert nr[1] / nr0[1] <= 1e-8 and ni[1] > 0


def test_mg_multi_follows_value_changes(binding):
    """After set_diagonal the multi-system V-cycle is still bitwise the
    single-system one (both read the problem's current matrix)."""
    P = binding.Problem.generate(32, 16, 24)
    try:
        n = P.nrow
        r = np.random.default_rng(5).standard_normal((4, n))
        for diag in (None, np.full(n, 30.0)):
            if diag is not None:
                P.set_diagonal(diag)
            z = np.zeros((4, n))
            P.ComputeMG_multi(r, z)
            for j in range(4):
                zj = np.zeros(n)
                P.ComputeMG(np.ascontiguousarray(r[j]), zj)
                assert np.array_equal(z[j], zj), (diag is None, j)
    finally:
        P.free()
