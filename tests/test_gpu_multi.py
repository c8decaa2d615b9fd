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


@pytest.mark.parametrize("lanes,bulk", [(1, 1), (2, 1), (4, 1), (2, 2), (4, 2), (2, 0)])
def test_every_multi_form_is_single_mg_bitwise(binding, monkeypatch, lanes, bulk):
    """Every (lanes, kernel form) of the eight-system path: register-pipelined,
    bulk-copy full phases and SpMV, bulk-copy first sweep too. Each system's
    V-cycle is bitwise the single-system one and the lockstep CG follows the
    single-system CG, on a grid whose coarse colour blocks start off tile
    boundaries (24 x 16 x 40)."""
    monkeypatch.setenv("HPCG_B200_MULTI_LANES", str(lanes))
    monkeypatch.setenv("HPCG_B200_MULTI_BULK", str(bulk))
    P = binding.Problem.generate(24, 16, 40)
    try:
        n = P.nrow
        r = np.random.default_rng(10 * lanes + bulk).standard_normal((8, n))
        z = np.zeros((8, n))
        P.ComputeMG_multi(r, z)
        for j in range(8):
            zj = np.zeros(n)
            P.ComputeMG(np.ascontiguousarray(r[j]), zj)
            assert np.array_equal(z[j], zj), j
        b = np.random.default_rng(5).uniform(-1.0, 1.0, (8, n))
        x = np.zeros((8, n))
        ni, nr, nr0 = P.CG_multi(b, x, 12, 0.0)
        for j in (0, 5):
            xs = np.zeros(n)
            ni_s, nr_s, nr0_s = P.CG(np.ascontiguousarray(b[j]), xs, 12, 0.0, True)
            s = nr_s / nr0_s
            assert ni[j] == ni_s == 12
            assert abs(nr[j] / nr0[j] - s) <= 1e-10 * max(s, 1e-9), (j, nr[j] / nr0[j], s)
    finally:
        P.free()
