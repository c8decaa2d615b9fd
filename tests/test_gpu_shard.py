"""The run over several ranks (hpcg_b200_generate_rank, hpcg_b200_comm_*,
hpcg_b200_shard_*) against the reference's own MPI code path.

The pin is the reference's MPI branch (SetupHalo_ref, ExchangeHalo,
ComputeDotProduct_ref's allreduce) compiled with the thread-based MPI stand-in of
oracle/mpi_shim (oracle/_ref/libhpcg_ref_mpi.so). Our ranks run on one GPU under a
local communicator, the same drivers a NCCL run uses.

* Each rank's right-hand side and every rank's SpMV are bitwise the reference's.
* Natural-order (level-scheduled) SYMGS and MG are bitwise the reference's on
  every rank: the halo is exchanged exactly where the reference exchanges it.
* Colour-order SYMGS/MG match the reference run on the colour-permuted ranks to
  1e-14 of max|x| (the last colour is not repeated at the turn of a sweep); CG
  histories match to |d| <= 1e-10 * max(r, 1e-9) on the scaled residual, dots to
  1e-13 relative (reductions are summed in a different order).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DECOMPS = [(1, 1, 2, 16, 16, 16), (2, 2, 2, 16, 16, 16), (3, 1, 2, 16, 8, 16)]


class Run:
    def __init__(self, oracle, binding, decomp, natural=False):
        if not oracle.have_reference_ranks():
            pytest.skip("oracle/_ref/libhpcg_ref_mpi.so missing")
        self.B = binding
        px, py, pz, nx, ny, nz = decomp
        self.decomp = decomp
        self.size = px * py * pz
        self.dims = (nx, ny, nz)
        self.P = [binding.Problem.generate_rank(nx, ny, nz, px, py, pz, r) for r in range(self.size)]
        if natural:
            for p in self.P:
                p.set_symgs_mode(binding.SYMGS_NATURAL)
        self.comm = binding.Comm.local(self.P)
        self.ref = oracle.ReferenceRanks(px, py, pz, nx, ny, nz)
        self.n = nx * ny * nz

    def perms(self):
        nx, ny, nz = self.dims
        return [self.B.colour_permutation(nx >> l, ny >> l, nz >> l)[0] for l in range(4)]

    def close(self):
        self.comm.free()
        for p in self.P:
            p.free()
        self.ref.close()


@pytest.fixture(scope="module", params=DECOMPS, ids=lambda d: "x".join(map(str, d[:3])))
def run(request, oracle, binding):
    R = Run(oracle, binding, request.param)
    yield R
    R.close()


@pytest.fixture(scope="module")
def run_natural(oracle, binding):
    R = Run(oracle, binding, DECOMPS[1], natural=True)
    yield R
    R.close()


def rand_vectors(run, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal(run.n) for _ in range(run.size)]


def test_rank_layout_and_rhs(run):
    for r, p in enumerate(run.P):
        info = p.rank_info(0)
        n, ncol = run.ref.sizes(r)[:2]
        assert info["rank"] == r and info["nranks"] == run.size
        assert info["externals"] == ncol - n
        assert np.array_equal(p.get_rhs(), run.ref.get_b(r))


def test_spmv_bitwise(run):
    xs = rand_vectors(run, 1)
    ys = [np.zeros(run.n) for _ in xs]
    run.comm.ComputeSPMV(xs, ys)
    for a, b in zip(ys, run.ref.spmv(xs)):
        assert np.array_equal(a, b)


def test_dot_allreduced(run):
    xs, ys = rand_vectors(run, 2), rand_vectors(run, 3)
    d = run.comm.ComputeDotProduct(xs, ys)
    ref = run.ref.dot(xs, ys)
    assert abs(d - ref) <= 1e-13 * max(abs(ref), 1.0)


def test_symgs_natural_bitwise(run_natural):
    R = run_natural
    rs, x0 = rand_vectors(R, 4), rand_vectors(R, 5)
    xs = [x.copy() for x in x0]
    R.comm.ComputeSYMGS(rs, xs)
    for a, b in zip(xs, R.ref.symgs(rs, x0)):
        assert np.array_equal(a, b)


def test_mg_natural_bitwise(run_natural):
    R = run_natural
    rs = rand_vectors(R, 6)
    zs = [np.zeros(R.n) for _ in rs]
    R.comm.ComputeMG(rs, zs)
    for a, b in zip(zs, R.ref.mg(rs)):
        assert np.array_equal(a, b)


def test_cg_natural_vs_reference(run_natural):
    R = run_natural
    bs = [R.ref.get_b(r) for r in range(R.size)]
    for it in (1, 10, 30):
        xs = [np.zeros(R.n) for _ in bs]
        ni, nr, nr0 = R.comm.CG(bs, xs, it, 0.0)
        xr, ni_r, nr_r, nr0_r = R.ref.cg(it, 0.0)
        assert ni == ni_r == it
        assert abs(nr0 - nr0_r) <= 1e-13 * nr0_r
        s = nr_r / nr0_r
        assert abs(nr / nr0 - s) <= 1e-10 * max(s, 1e-9), (it, nr / nr0, s)
        for a, b in zip(xs, xr):
            assert np.max(np.abs(a - b)) <= 1e-9 * max(np.max(np.abs(b)), 1.0)


@pytest.fixture(scope="module")
def run_colour_ref(oracle, binding):
    """Colour-order ranks next to the reference run on the colour-permuted ranks."""
    R = Run(oracle, binding, DECOMPS[1])
    perms = R.perms()
    for r in range(R.size):
        R.ref.permute(r, perms)
    yield R, perms[0]
    R.close()


def test_symgs_mg_colour_vs_permuted_reference(run_colour_ref):
    R, n2o = run_colour_ref
    rs, x0 = rand_vectors(R, 7), rand_vectors(R, 8)
    xs = [x.copy() for x in x0]
    R.comm.ComputeSYMGS(rs, xs)
    ref = R.ref.symgs([r[n2o] for r in rs], [x[n2o] for x in x0])
    for a, bc in zip(xs, ref):
        b = np.empty_like(bc)
        b[n2o] = bc
        assert np.max(np.abs(a - b)) <= 1e-14 * np.max(np.abs(b))
    zs = [np.zeros(R.n) for _ in rs]
    R.comm.ComputeMG(rs, zs)
    ref = R.ref.mg([r[n2o] for r in rs])
    for a, bc in zip(zs, ref):
        b = np.empty_like(bc)
        b[n2o] = bc
        assert np.max(np.abs(a - b)) <= 1e-14 * np.max(np.abs(b))


def test_cg_colour_vs_permuted_reference(run_colour_ref):
    R, n2o = run_colour_ref
    bs = [R.P[r].get_rhs() for r in range(R.size)]
    for it in (1, 10, 30):
        xs = [np.zeros(R.n) for _ in bs]
        ni, nr, nr0 = R.comm.CG(bs, xs, it, 0.0)
        xr, ni_r, nr_r, nr0_r = R.ref.cg(it, 0.0)
        assert ni == ni_r == it
        s = nr_r / nr0_r
        assert abs(nr / nr0 - s) <= 1e-10 * max(s, 1e-9), (it, nr / nr0, s)


def test_bulk_config_ranks_vs_permuted_reference(oracle, binding, monkeypatch):
    """The bulk-copy pipeline (configuration 10) on ranks with halos (3 x 1 x 2,
    odd coarse blocks): colour MG as the reference run on the colour-permuted
    ranks, and the CG history as before."""
    monkeypatch.setenv("HPCG_B200_CONFIG", "10")
    R = Run(oracle, binding, DECOMPS[2])
    try:
        n2o = R.perms()[0]
        perms = R.perms()
        for r in range(R.size):
            R.ref.permute(r, perms)
        rs = rand_vectors(R, 12)
        zs = [np.zeros(R.n) for _ in rs]
        R.comm.ComputeMG(rs, zs)
        assert R.P[0].level_config(0)["gs"] == 10
        ref = R.ref.mg([r[n2o] for r in rs])
        for a, bc in zip(zs, ref):
            b = np.empty_like(bc)
            b[n2o] = bc
            assert np.max(np.abs(a - b)) <= 1e-14 * np.max(np.abs(b))
        bs = [p.get_rhs() for p in R.P]
        xs = [np.zeros(R.n) for _ in bs]
        ni, nr, nr0 = R.comm.CG(bs, xs, 10, 0.0)
        xr, ni_r, nr_r, nr0_r = R.ref.cg(10, 0.0)
        s_ = nr_r / nr0_r
        assert ni == ni_r == 10 and abs(nr / nr0 - s_) <= 1e-10 * max(s_, 1e-9)
    finally:
        R.close()


def test_cg_converges_and_tolerance_stop(run):
    bs = [p.get_rhs() for p in run.P]
    xs = [np.zeros(run.n) for _ in bs]
    ni, nr, nr0 = run.comm.CG(bs, xs, 500, 1e-9)
    assert nr / nr0 <= 1e-9 and 0 < ni < 500
    # the exact solution of HPCG's system is all ones (GenerateProblem_ref.cpp:178-181)
    for x in xs:
        assert np.max(np.abs(x - 1.0)) < 1e-6


def test_cg_times_slots(run):
    """times[0..5] as CG.cpp:132-139 files them, from the sharded driver on the
    local communicator (no MPI, one GPU): every slot positive, the allreduce
    step (times[4]) inside the dot-product time (times[1]), and the four
    disjoint parts (dots, updates, SpMV, preconditioner) together within the
    whole call (times[0]). Accumulates over calls, as the reference's slots do."""
    bs = [p.get_rhs() for p in run.P]
    xs = [np.zeros(run.n) for _ in bs]
    t = np.zeros(10)
    run.comm.CG(bs, xs, 10, 0.0, times=t)
    assert np.all(t[:6] > 0.0), t
    assert t[4] <= t[1]
    assert t[1] + t[2] + t[3] + t[5] <= t[0]
    assert np.all(t[6:] == 0.0)
    t1 = t.copy()
    xs = [np.zeros(run.n) for _ in bs]
    run.comm.CG(bs, xs, 10, 0.0, times=t)
    assert np.all(t[:6] > t1[:6])


def test_device_vectors(run):
    import torch
    xs = rand_vectors(run, 9)
    ys_host = [np.zeros(run.n) for _ in xs]
    run.comm.ComputeSPMV(xs, ys_host)
    xd = [torch.from_numpy(x).cuda() for x in xs]
    yd = [torch.zeros(run.n, dtype=torch.float64, device="cuda") for _ in xs]
    run.comm.ComputeSPMV(xd, yd)
    for a, b in zip(yd, ys_host):
        assert np.array_equal(a.cpu().numpy(), b)


def test_single_rank_entry_points_refuse_a_rank(run, binding):
    p = run.P[0]
    x = np.zeros(run.n)
    with pytest.raises(binding.HpcgError) as e:
        p.CG(p.get_rhs(), x, 5, 0.0)
    assert e.value.status == binding.ERR_UNSUPPORTED
    with pytest.raises(binding.HpcgError):
        p.ComputeSPMV(x, x.copy())


def test_local_comm_rejects_wrong_rank_order(binding):
    P = [binding.Problem.generate_rank(8, 8, 8, 2, 1, 1, r) for r in range(2)]
    try:
        with pytest.raises(binding.HpcgError):
            binding.Comm.local([P[1], P[0]])
        with pytest.raises(binding.HpcgError):
            binding.Comm.local([P[0]])
    finally:
        for p in P:
            p.free()


def test_far_halo_columns_stay_unpacked(binding):
    """A rank's external columns follow its n interior rows, so on a 48^3 rank
    with a neighbour a 128-row tile of level 0 mixes interior columns with
    external ones more than 65534 apart: that level keeps its 32-bit columns,
    and the coarser levels, whose columns fit one of the packed forms, are
    packed."""
    P = binding.Problem.generate_rank(48, 48, 48, 2, 1, 1, 0)
    try:
        assert P.level_packed(0) == 0
        for lv in (1, 2, 3):
            _, pitch, _ = P.level_info(lv)
            assert P.level_packed(lv) in (pitch // 128 * 3568, pitch // 128 * 7024, pitch // 128 * 544)
    finally:
        P.free()


@pytest.mark.parametrize("cfg", ["1", "10"])
def test_nccl_single_rank_equals_single_gpu_cg(binding, monkeypatch, cfg):
    """A one-rank NCCL communicator (NCCL opened, initialised and allreducing on
    the GPU) runs the sharded driver; it equals hpcg_b200_cg bit for bit.
    Both problems run the same kernel configuration: the r'z fused into the
    post-smoother sums one partial per block, so its rounding follows the grid
    of the configuration the tuner picks, and two problems tuned apart may
    differ in the last bits of the residual."""
    monkeypatch.setenv("HPCG_B200_CONFIG", cfg)
    uid = binding.comm_unique_id()
    P = binding.Problem.generate_rank(16, 16, 16, 1, 1, 1, 0)
    S = binding.Problem.generate(16)
    C = binding.Comm.nccl(uid, 1, 0, P)
    try:
        b = S.get_rhs()
        x1 = np.zeros(S.nrow)
        x2 = np.zeros(S.nrow)
        r1 = S.CG(b, x1, 20, 0.0)
        r2 = C.CG([b], [x2], 20, 0.0)
        assert r1 == r2
        assert np.array_equal(x1, x2)
        # the NCCL allreduce is timed into times[4], inside the dot time
        t = np.zeros(10)
        x3 = np.zeros(S.nrow)
        assert C.CG([b], [x3], 20, 0.0, times=t) == r1
        assert np.all(t[:6] > 0.0) and t[4] <= t[1] and t[1] + t[2] + t[3] + t[5] <= t[0], t
        assert C.ComputeDotProduct([b], [b]) == binding.ComputeDotProduct(S.nrow, b, b)
    finally:
        C.free()
        P.free()
        S.free()
