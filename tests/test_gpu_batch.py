"""Batched solves (hpcg_b200_batch_*): problems of different sizes advanced
together must follow their one-at-a-time solves (hpcg_b200_cg_mixed): the same
V-cycle bits per problem, dots in another (fixed) order, so the same iteration
counts within one, scaled residuals within 1e-10 * max(r, 1e-9) on fixed
iteration counts, and solutions within 1e-7 at the tolerance. The one-launch
iteration (every step in one cooperative launch) equals the launch-per-step
form on the register phases bit for bit, and its grid barrier's bounded wait
ends by itself."""
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


def test_batch_one_launch_iteration_equals_launch_per_step(binding, monkeypatch):
    """The whole iteration as one cooperative launch (steps separated by grid
    barriers) computes the same bits as one launch per step on the register
    phases: the same work lists, the same per-tile partials, the same order.
    Compared on fixed iteration counts and at a tolerance, with a problem that
    converges early (zero right-hand side)."""
    dims = [(16, 32, 48), (32, 16, 16), (16, 16, 16)]
    outs = []
    for persist in ("1", "0"):
        monkeypatch.setenv("HPCG_B200_BATCH_PERSIST", persist)
        monkeypatch.setenv("HPCG_B200_BATCH_BULK", "0")
        B = binding.Batch(dims)
        try:
            assert B.form() == (2 if persist == "1" else 0)
            bs = [p.get_rhs() for p in B.problems]
            bs[2] = np.zeros_like(bs[2])
            res = []
            for iters, tol in ((7, 0.0), (500, 1e-9)):
                xs = [np.zeros(p.nrow) for p in B.problems]
                ni, nr, nr0 = B.CG_mixed(bs, xs, iters, tol)
                res.append((ni.copy(), nr.copy(), nr0.copy(), [x.copy() for x in xs]))
            outs.append(res)
        finally:
            B.free()
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
        for xa, xb in zip(a[3], b[3]):
            assert np.array_equal(xa, xb)
    assert outs[0][1][0][2] == 0 and np.all(outs[0][1][1][:2] / outs[0][1][2][:2] <= 1e-9)


def test_grid_barrier_wait_gives_up_and_context_survives(binding, monkeypatch):
    """The grid barrier of the one-launch iteration ends by itself: with one
    arrival more expected than the grid holds, every block's wait gives up
    after the limit and the call returns HPCG_B200_ERR_TIMEOUT; the same context
    then runs a batched solve in the one-launch form."""
    import time
    t0 = time.perf_counter()
    st = binding.grid_wait_selftest(0.25)
    dt = time.perf_counter() - t0
    assert st == binding.ERR_TIMEOUT
    assert 0.2 <= dt < 30.0
    assert "gave up" in binding.last_error()
    monkeypatch.setenv("HPCG_B200_BATCH_PERSIST", "1")
    B = binding.Batch([(16, 16, 32), (32, 16, 16)])
    try:
        assert B.form() == 2
        bs = [p.get_rhs() for p in B.problems]
        xs = [np.zeros(p.nrow) for p in B.problems]
        ni, nr, nr0 = B.CG_mixed(bs, xs, 200, 1e-8)
        assert np.all(nr / nr0 <= 1e-8)
    finally:
        B.free()
