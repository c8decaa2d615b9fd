"""Batched solves (hpcg_b200_batch_*): problems of different sizes advanced
together must follow their one-at-a-time solves (hpcg_b200_cg_mixed): the same
V-cycle bits per problem, dots in another (fixed) order, so the same iteration
counts within one, scaled residuals within 1e-10 * max(r, 1e-9) on fixed
iteration counts, and solutions within 1e-7 at the tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIMS = [(32, 32, 32), (48, 32, 16), (16, 16, 16), (32, 64, 48)]


@pytest.fixture(scope="module")
def batch(binding):
    B = binding.Batch(DIMS)
    yield B
    B.free()


def test_batch_fixed_iterations_follow_single_solves(batch):
    bs = [p.get_rhs() for p in batch.problems]
    for iters in (1, 6):
        xs = [np.zeros(p.nrow) for p in batch.problems]
        ni, nr, nr0 = batch.CG_mixed(bs, xs, iters, 0.0)
        for i, p in enumerate(batch.problems):
            x1 = np.zeros(p.nrow)
            n1, r1, r01 = p.CG_mixed(bs[i], x1, iters, 0.0)
            assert ni[i] == n1 == iters
            assert abs(nr0[i] - r01) <= 1e-13 * r01
            s = r1 / r01
            assert abs(nr[i] / nr0[i] - s) <= 1e-10 * max(s, 1e-9), (i, nr[i] / nr0[i], s)
            assert np.max(np.abs(xs[i] - x1)) <= 1e-9 * max(np.max(np.abs(x1)), 1.0)


def test_batch_to_tolerance(batch):
    rng = np.random.Generator(np.random.PCG64(11))
    bs = [rng.uniform(-1.0, 1.0, p.nrow) for p in batch.problems]
    xs = [np.zeros(p.nrow) for p in batch.problems]
    ni, nr, nr0 = batch.CG_mixed(bs, xs, 500, 1e-9)
    for i, p in enumerate(batch.problems):
        assert nr[i] / nr0[i] <= 1e-9
        x1 = np.zeros(p.nrow)
        n1, r1, r01 = p.CG_mixed(bs[i], x1, 500, 1e-9)
        assert abs(int(ni[i]) - n1) <= 1
        assert np.linalg.norm(xs[i] - x1) <= 1e-7 * np.linalg.norm(x1)


def test_batch_device_vectors_and_errors(binding, batch):
    import torch
    bs = [torch.from_numpy(p.get_rhs()).cuda() for p in batch.problems]
    xs = [torch.zeros_like(b) for b in bs]
    ni, nr, nr0 = batch.CG_mixed(bs, xs, 200, 1e-8)
    assert np.all(nr / nr0 <= 1e-8)
    with pytest.raises(binding.HpcgError) as e:
        binding.Batch([(24, 24, 24)])
    assert e.value.status == binding.ERR_UNSUPPORTED


@pytest.mark.parametrize("bulk", ["0", "1"])
def test_batch_both_phase_kernels_follow_single_solves(binding, monkeypatch, bulk):
    """The batched colour phases on the 256-row register kernel and on the
    bulk-copy kernel (128-row blocks of each problem's blocked FP32 copy, the
    tiles of converged problems skipped): each follows its one-at-a-time solve,
    including a problem that converges early (zero right-hand side)."""
    monkeypatch.setenv("HPCG_B200_BATCH_BULK", bulk)
    B = binding.Batch([(16, 32, 48), (32, 16, 16), (16, 16, 16)])
    try:
        bs = [p.get_rhs() for p in B.problems]
        bs[2] = np.zeros_like(bs[2])
        xs = [np.zeros(p.nrow) for p in B.problems]
        ni, nr, nr0 = B.CG_mixed(bs, xs, 8, 0.0)
        assert ni[2] == 0 and nr0[2] == 0.0
        for i in (0, 1):
            p = B.problems[i]
            x1 = np.zeros(p.nrow)
            n1, r1, r01 = p.CG_mixed(bs[i], x1, 8, 0.0)
            assert ni[i] == n1 == 8
            s = r1 / r01
            assert abs(nr[i] / nr0[i] - s) <= 1e-10 * max(s, 1e-9), (i, nr[i] / nr0[i], s)
            assert np.max(np.abs(xs[i] - x1)) <= 1e-9 * max(np.max(np.abs(x1)), 1.0)
    finally:
        B.free()
