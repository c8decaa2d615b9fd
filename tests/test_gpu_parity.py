"""Parity of the CUDA path with the oracle, through the C ABI (needs a B200).

Tolerances. The row kernels (SpMV, Gauss-Seidel, restriction, prolongation,
WAXPBY) use the reference's operation order without contraction, so their
results are compared bit for bit (np.array_equal, which counts -0.0 == 0.0).
The colour-ordered symmetric Gauss-Seidel does not repeat the last colour at
the turn of the sweep; it is bitwise equal to the oracle's ora_symgs_skip and
within 1e-14 (relative to max |x|) of ComputeSYMGS_ref on the same ordering.
Dot products reduce in a fixed tree instead of a serial loop: relative 1e-13.
CG residual histories: |ours - reference| <= 1e-10 * max(reference, 1e-9) on the
scaled residual (below 1e-9 the history is dominated by rounding).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def levels_of(P):
    return [dict(nx=L.nx, ny=L.ny, nz=L.nz, nnz=L.nnz, cols=L.cols, vals=L.vals, f2c=L.f2c) for L in P.levels]


def perms_of(binding, P):
    return [binding.colour_permutation(L.nx, L.ny, L.nz)[0] for L in P.levels]


def skip_of(binding, P):
    """Rows of the last colour block of each level (not repeated at the turn of a sweep)."""
    out = []
    for L in P.levels:
        st = binding.colour_permutation(L.nx, L.ny, L.nz)[1]
        last = max(s for s in range(8) if st[s + 1] > st[s])
        out.append(int(st[last + 1] - st[last]))
    return out


@pytest.fixture(scope="module")
def case16(oracle, binding):
    P = oracle.generate(16)
    D = binding.Problem.optimize(levels_of(P))
    perms = perms_of(binding, P)
    yield P, D, perms, oracle.permute(P.levels, perms)
    D.free()


@pytest.fixture(scope="module")
def case32(oracle, binding):
    P = oracle.generate(32)
    D = binding.Problem.optimize(levels_of(P))
    perms = perms_of(binding, P)
    yield P, D, perms, oracle.permute(P.levels, perms)
    D.free()


def hist_close(a, b, rel=1e-10):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    bound = rel * np.maximum(np.abs(b), 1e-9)
    assert np.all(np.abs(a - b) <= bound), (a, b, np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


# ---------------------------------------------------------------------------
# layout
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("dims", [(16, 16, 16), (16, 24, 32), (24, 24, 24)])
def test_layout_matches_reference_structures(oracle, binding, dims):
    P = oracle.generate(*dims)
    D = binding.Problem.optimize(levels_of(P))
    try:
        for l, L in enumerate(P.levels):
            E = D.export_level(l)
            n2o, starts = binding.colour_permutation(L.nx, L.ny, L.nz)
            assert np.array_equal(E["new2old"], n2o) and np.array_equal(E["starts"], starts)
            o2n = np.empty_like(n2o)
            o2n[n2o] = np.arange(L.n, dtype=np.int32)
            cols, vals = L.dense_rows()
            exp_c = np.full((27, L.n), L.n, np.int32)
            exp_v = np.zeros((27, L.n))
            for i in range(L.n):
                q = o2n[i]
                iz, rem = divmod(i, L.nx * L.ny)
                iy, ix = divmod(rem, L.nx)
                for j in range(L.nnz[i]):
                    c = cols[i, j]
                    cz, r2 = divmod(c, L.nx * L.ny)
                    cy, cx = divmod(r2, L.nx)
                    k = (cz - iz + 1) * 9 + (cy - iy + 1) * 3 + (cx - ix + 1)
                    exp_c[k, q] = o2n[c]
                    exp_v[k, q] = vals[i, j]
            assert np.array_equal(E["cols"][:, : L.n], exp_c)
            assert np.array_equal(E["vals"][:, : L.n], exp_v)
            if L.f2c is not None:
                nc = P.levels[l + 1]
                c_n2o = binding.colour_permutation(nc.nx, nc.ny, nc.nz)[0]
                assert np.array_equal(E["f2c"], o2n[L.f2c[c_n2o]])
    finally:
        D.free()


@pytest.mark.parametrize("dims", [(16, 16, 16), (16, 24, 32), (24, 24, 24), (32, 32, 32)])
def test_device_generator_equals_optimize(oracle, binding, dims):
    """hpcg_b200_generate builds on the device what OptimizeProblem builds from
    the reference's host structures (GenerateProblem_ref + GenerateCoarseProblem)."""
    P = oracle.generate(*dims)
    A = binding.Problem.optimize(levels_of(P))
    G = binding.Problem.generate(*dims)
    try:
        for l, L in enumerate(P.levels):
            a, g = A.export_level(l), G.export_level(l)
            n = a["n"]
            for key in ("new2old", "starts"):
                assert np.array_equal(a[key], g[key])
            assert np.array_equal(a["cols"][:, :n], g["cols"][:, :n])
            assert np.array_equal(a["vals"][:, :n], g["vals"][:, :n])
            if a["f2c"] is not None:
                assert np.array_equal(a["f2c"], g["f2c"])
        assert np.array_equal(G.get_rhs(), P.b)
        assert G.memory_use() > 0
    finally:
        A.free()
        G.free()


# ---------------------------------------------------------------------------
# row kernels: bitwise
# ---------------------------------------------------------------------------

def test_spmv_bitwise(oracle, case32):
    P, D, _, _ = case32
    rng = np.random.default_rng(11)
    for x in (rng.random(P.levels[0].n), rng.standard_normal(P.levels[0].n), P.xexact):
        y = np.zeros_like(x)
        assert D.ComputeSPMV(x, y) == 0
        assert np.array_equal(y, oracle.spmv(P.levels[0], x))
    # A * xexact = b exactly (b_i = 27 - nnz_i, GenerateProblem_ref.cpp:178)
    y = np.zeros(P.levels[0].n)
    D.ComputeSPMV(P.xexact, y)
    assert np.array_equal(y, P.b)


@pytest.mark.parametrize("order", [0, 1, 2])
def test_spmv_every_row_order_bitwise(oracle, binding, monkeypatch, order):
    """Every row order of the SpMV (storage, natural, slab) computes the
    reference's bits on a 32 x 24 x 48 grid; the CG's fused p'Ap variant runs in each."""
    monkeypatch.setenv("HPCG_B200_SPMV_ORDER", str(order))
    L = oracle.generate(32, 24, 48).levels
    D = binding.Problem.generate(32, 24, 48)
    try:
        x = np.random.default_rng(order).standard_normal(L[0].n)
        y = np.zeros_like(x)
        D.ComputeSPMV(x, y)
        assert D.level_config(0)["spmv_order"] == order
        assert np.array_equal(y, oracle.spmv(L[0], x))
        b = D.get_rhs()
        x1 = np.zeros_like(b)
        D.CG(b, x1, 3, 0.0)  # the fused p'Ap path in this order
        assert np.all(np.isfinite(x1))
    finally:
        D.free()


@pytest.mark.parametrize("dims,order", [((32, 16, 24), 2), ((32, 24, 48), 0), ((32, 24, 48), 2)])
def test_bulk_spmv_and_phases_vs_oracle(oracle, binding, monkeypatch, dims, order):
    """SpMV configuration 7 (tiles streamed by tensor copies; slab order where the
    slab runs split into 128-row tiles, 32 x 16 x 24, else storage order) and
    the bulk Gauss-Seidel phases on every level, set through
    HPCG_B200_LEVEL_CONFIG: SpMV bitwise the reference's, CG (fused p'Ap and
    r'z partials) as the oracle's on the colour order."""
    cfg = ";".join(["10,10,7,%d,10,10" % order] * 4)
    monkeypatch.setenv("HPCG_B200_LEVEL_CONFIG", cfg)
    P = oracle.generate(*dims)
    D = binding.Problem.optimize(levels_of(P))
    try:
        x = np.random.default_rng(order).standard_normal(P.levels[0].n)
        y = np.zeros_like(x)
        D.ComputeSPMV(x, y)  # first use: the configurations are set here
        for l in range(4):
            c = D.level_config(l)
            assert (c["gs"], c["gs_first"], c["spmv"], c["spmv_order"]) == (10, 10, 7, order)
        assert np.array_equal(y, oracle.spmv(P.levels[0], x))
        perms = perms_of(binding, P)
        PL = oracle.permute(P.levels, perms)
        for k in (1, 10, 30):
            xs = np.zeros(P.levels[0].n)
            ni, nr, nr0 = D.CG(P.b, xs, k, 0.0, True)
            xo, nio, nro, nr0o, _ = oracle.cg(PL, P.b[perms[0]], np.zeros(P.levels[0].n), k, 0.0,
                                              skip=skip_of(binding, P))
            assert ni == nio == k
            hist_close([nr / nr0], [nro / nr0o])
    finally:
        D.free()


def test_level_config_override_rejects_bad_values(binding, monkeypatch):
    """A malformed or out-of-range HPCG_B200_LEVEL_CONFIG is ignored (the level is tuned)."""
    monkeypatch.setenv("HPCG_B200_LEVEL_CONFIG", "10,5,99,2,10,5")
    D = binding.Problem.generate(16)
    try:
        x = np.zeros(16 ** 3)
        D.ComputeSPMV(x, x.copy())
        c = D.level_config(0)
        assert c["tuned"] == 1 and c["spmv"] < 8
    finally:
        D.free()


def test_level_config_override_per_position(binding, monkeypatch):
    """HPCG_B200_LEVEL_CONFIG's first-sweep fields may give one configuration
    per sweep position; hpcg_b200_level_first_config reports them, and the
    string the binding builds from a tuned problem sets the same choices."""
    monkeypatch.setenv("HPCG_B200_LEVEL_CONFIG", "10,1/2/3/4/5/6/7/10,7,0,10,5;1,1,1,0,1,1;1,1,1,0,1,1;1,1,1,0,1,1")
    D = binding.Problem.generate(32)
    try:
        x = np.zeros(32 ** 3)
        D.ComputeMG(x, x.copy())
        f64, f32 = D.level_first_config(0)
        assert f64 == [1, 2, 3, 4, 5, 6, 7, 10]
        assert D.level_config(0)["gs_first"] == 1 and D.level_first_config(1)[0] == [1] * 8
    finally:
        D.free()
    monkeypatch.delenv("HPCG_B200_LEVEL_CONFIG")
    T = binding.Problem.generate(32)
    try:
        y = np.zeros(32 ** 3)
        T.ComputeMG(y, y.copy())
        T.CG_mixed(y, y.copy(), 1, 0.0)
        s = T.level_config_string()
        monkeypatch.setenv("HPCG_B200_LEVEL_CONFIG", s)
        R = binding.Problem.generate(32)
        try:
            R.ComputeMG(y, y.copy())
            R.CG_mixed(y, y.copy(), 1, 0.0)
            assert R.level_config_string() == s
        finally:
            R.free()
    finally:
        T.free()


def test_spmv_matches_reference_golden(oracle, case16):
    P, D, _, _ = case16
    g = np.load(os.path.join(GOLD, "golden_16.npz"))
    y = np.zeros(16 ** 3)
    D.ComputeSPMV(g["x_seed"], y)
    assert np.array_equal(y, g["spmv"])


def test_symgs_colour_bitwise(oracle, binding, case32):
    P, D, perms, PL = case32
    rng = np.random.default_rng(12)
    r, x0 = rng.standard_normal(P.levels[0].n), rng.standard_normal(P.levels[0].n)
    x = x0.copy()
    D.set_symgs_mode(binding.SYMGS_COLOUR)
    D.ComputeSYMGS(r, x)
    p0 = perms[0]
    exp = np.empty_like(x)
    exp[p0] = oracle.symgs_skip(PL[0], r[p0], x0[p0], skip_of(binding, P)[0])
    assert np.array_equal(x, exp)
    ref = np.empty_like(x)
    ref[p0] = oracle.symgs(PL[0], r[p0], x0[p0])
    assert np.max(np.abs(x - ref)) <= 1e-14 * np.max(np.abs(ref))


def test_symgs_natural_is_reference_bitwise(oracle, binding, case16):
    """The level-scheduled mode reproduces ComputeSYMGS_ref's natural-order sweep."""
    P, D, _, _ = case16
    g = np.load(os.path.join(GOLD, "golden_16.npz"))
    D.set_symgs_mode(binding.SYMGS_NATURAL)
    try:
        x = g["x_seed"].copy()
        D.ComputeSYMGS(g["b"], x)
        assert np.array_equal(x, g["symgs"])
        rng = np.random.default_rng(13)
        r, x0 = rng.standard_normal(16 ** 3), rng.standard_normal(16 ** 3)
        x = x0.copy()
        D.ComputeSYMGS(r, x)
        assert np.array_equal(x, oracle.symgs(P.levels[0], r, x0))
    finally:
        D.set_symgs_mode(binding.SYMGS_COLOUR)


def test_mg_colour_bitwise(oracle, binding, case32):
    P, D, perms, PL = case32
    r = np.random.default_rng(14).standard_normal(P.levels[0].n)
    z = np.zeros_like(r)
    D.ComputeMG(r, z)
    p0 = perms[0]
    exp = np.empty_like(z)
    exp[p0] = oracle.mg(PL, r[p0], skip=skip_of(binding, P))
    assert np.array_equal(z, exp)
    ref = np.empty_like(z)
    ref[p0] = oracle.mg(PL, r[p0])
    assert np.max(np.abs(z - ref)) <= 1e-14 * np.max(np.abs(ref))


@pytest.mark.parametrize("cfg", [str(c) for c in range(11)])
def test_mg_colour_every_config_bitwise(oracle, binding, monkeypatch, cfg):
    """Every kernel configuration of the phases (load schedules, registers, 2 or 4
    contiguous rows with vector loads, 2 or 4 interleaved rows, shared-memory
    tiles filled by asynchronous copies, the bulk-copy pipeline) computes the same
    V-cycle bits; the coarsest level (3 x 2 x 5) has colour blocks of odd sizes
    starting off multiples of 4."""
    monkeypatch.setenv("HPCG_B200_CONFIG", cfg)
    P = oracle.generate(24, 16, 40)
    D = binding.Problem.generate(24, 16, 40)
    try:
        perms = perms_of(binding, P)
        PL = oracle.permute(P.levels, perms)
        r = np.random.default_rng(int(cfg)).standard_normal(P.levels[0].n)
        z = np.zeros_like(r)
        D.ComputeMG(r, z)
        assert D.level_config(0)["gs"] == int(cfg)
        exp = np.empty_like(z)
        exp[perms[0]] = oracle.mg(PL, r[perms[0]], skip=skip_of(binding, P))
        assert np.array_equal(z, exp)
    finally:
        D.free()


def test_mg_natural_is_reference_bitwise(oracle, binding, case16):
    P, D, _, _ = case16
    g = np.load(os.path.join(GOLD, "golden_16.npz"))
    D.set_symgs_mode(binding.SYMGS_NATURAL)
    try:
        z = np.zeros(16 ** 3)
        D.ComputeMG(g["x_seed"], z)
        assert np.array_equal(z, g["mg"])
    finally:
        D.set_symgs_mode(binding.SYMGS_COLOUR)


def test_mg_repeat_is_identical(case32):
    """Stale work vectors never leak into a V-cycle: two calls give the same bits."""
    P, D, _, _ = case32
    rng = np.random.default_rng(15)
    r1, r2 = rng.standard_normal(P.levels[0].n), rng.standard_normal(P.levels[0].n)
    a = np.zeros_like(r1)
    D.ComputeMG(r1, a)
    b_ = np.zeros_like(r1)
    D.ComputeMG(r2, b_)
    c = np.zeros_like(r1)
    D.ComputeMG(r1, c)
    assert np.array_equal(a, c)


# ---------------------------------------------------------------------------
# vector routines
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("n", [1, 7, 1000, 32768, 1 << 20])
def test_dot_waxpby_residual(oracle, binding, n):
    rng = np.random.default_rng(n)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    d = binding.ComputeDotProduct(n, x, y)
    ref = oracle.dot(x, y)
    assert abs(d - ref) <= 1e-13 * max(abs(ref), np.abs(x * y).sum() * 1e-3)
    assert binding.ComputeDotProduct(n, x, y) == d  # deterministic
    assert binding.ComputeDotProduct(n, x, x) == pytest.approx(oracle.dot(x, x), rel=1e-13)
    for alpha, beta in ((1.0, 2.5), (0.75, 1.0), (-1.5, 0.25), (1.0, 0.0)):
        w = np.zeros(n)
        binding.ComputeWAXPBY(n, alpha, x, beta, y, w)
        assert np.array_equal(w, oracle.waxpby(alpha, x, beta, y))
    assert binding.ComputeResidual(n, x, y) == oracle.residual(x, y)


def test_zero_length_and_aliasing(binding):
    x = np.arange(5.0)
    assert binding.ComputeDotProduct(0, x, x) == 0.0
    w = x.copy()
    binding.ComputeWAXPBY(5, 2.0, w, 1.0, w, w)  # in place, x == y == w
    assert np.array_equal(w, 3.0 * x)


def test_device_pointers_match_host(oracle, binding, case32):
    import torch
    P, D, _, _ = case32
    n = P.levels[0].n
    x = np.random.default_rng(16).standard_normal(n)
    yh = np.zeros(n)
    D.ComputeSPMV(x, yh)
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros(n, dtype=torch.float64, device="cuda")
    D.ComputeSPMV(xd, yd)
    torch.cuda.synchronize()
    assert np.array_equal(yd.cpu().numpy(), yh)
    zh = np.zeros(n)
    D.ComputeMG(x, zh)
    zd = torch.zeros(n, dtype=torch.float64, device="cuda")
    D.ComputeMG(xd, zd)
    assert np.array_equal(zd.cpu().numpy(), zh)
    assert binding.ComputeDotProduct(n, xd, yd) == binding.ComputeDotProduct(n, x, yh)


# ---------------------------------------------------------------------------
# CG
# ---------------------------------------------------------------------------

def test_cg_colour_history_vs_reference_on_permuted_system(oracle, binding, case16):
    """History against CG_ref run by the reference itself on the colour-permuted
    hierarchy (golden_16.npz cg_hist_perm)."""
    P, D, perms, PL = case16
    g = np.load(os.path.join(GOLD, "golden_16.npz"))
    ours = []
    for k in range(1, 21):
        x = np.zeros(16 ** 3)
        ni, nr, nr0 = D.CG(P.b, x, k, 0.0, True)
        assert ni == k
        ours.append(nr / nr0)
    hist_close(ours, g["cg_hist_perm"])


def oracle_binding():
    from hpcg_b200 import binding
    return binding


def test_cg_colour_vs_oracle_32(oracle, case32):
    P, D, perms, PL = case32
    b = P.b[perms[0]]
    for k in (1, 5, 10, 25, 50):
        x = np.zeros(32 ** 3)
        ni, nr, nr0 = D.CG(P.b, x, k, 0.0, True)
        xo, nio, nro, nr0o, _ = oracle.cg(PL, b, np.zeros(32 ** 3), k, 0.0, skip=skip_of(oracle_binding(), P))
        assert ni == nio == k
        assert abs(nr0 - nr0o) <= 1e-13 * nr0o
        hist_close([nr / nr0], [nro / nr0o])
        xn = np.empty_like(xo)
        xn[perms[0]] = xo
        assert np.max(np.abs(x - xn)) <= 1e-10 * max(np.max(np.abs(xn)), 1.0)


def test_cg_natural_is_reference(oracle, binding, case16):
    """Natural-order SYMGS: the whole CG is CG_ref except for the dot reductions."""
    P, D, _, _ = case16
    g = np.load(os.path.join(GOLD, "golden_16.npz"))
    D.set_symgs_mode(binding.SYMGS_NATURAL)
    try:
        ours = []
        for k in (1, 2, 5, 10, 20):
            x = np.zeros(16 ** 3)
            ni, nr, nr0 = D.CG(P.b, x, k, 0.0, True)
            ours.append(nr / nr0)
            assert nr0 == pytest.approx(float(g["normr0"]), rel=1e-14)
            if k == 10:
                assert np.max(np.abs(x - g["cg_x10"])) <= 1e-12
        hist_close(ours, g["cg_hist"][[0, 1, 4, 9, 19]])
    finally:
        D.set_symgs_mode(binding.SYMGS_COLOUR)


def test_cg_tolerance_stop_and_unpreconditioned(oracle, case32):
    P, D, perms, PL = case32
    b = P.b[perms[0]]
    for prec in (True, False):
        x = np.zeros(32 ** 3)
        ni, nr, nr0 = D.CG(P.b, x, 500, 1e-8, prec)
        _, nio, nro, nr0o, _ = oracle.cg(PL, b, np.zeros(32 ** 3), 500, 1e-8, prec)
        assert ni == nio
        assert nr / nr0 <= 1e-8


def test_cg_reproducible_testnorms(case32):
    """TestNorms (src/TestNorms.cpp:31-46) needs the scaled residual of repeated
    sets to vary < 1e-6; the fixed reduction order makes it identical."""
    P, D, _, _ = case32
    vals = []
    for _ in range(3):
        x = np.zeros(32 ** 3)
        ni, nr, nr0 = D.CG(P.b, x, 50, 0.0, True)
        vals.append(nr / nr0)
    assert vals[0] == vals[1] == vals[2]


def test_testcg_exaggerated_diagonal(oracle, binding):
    """TestCG.cpp:52-123 on the device: the diagonal is rewritten through
    ReplaceMatrixDiagonal on the host, resent with hpcg_b200_set_diagonal; CG
    converges in <= 12 unpreconditioned and <= 2 preconditioned iterations."""
    P = oracle.generate(32)
    D = binding.Problem.optimize(levels_of(P))
    try:
        n = P.levels[0].n
        diag = np.full(n, 26.0)
        scale = np.full(n, 1.0e6)
        scale[:9] = (np.arange(9) + 2) * 1.0e6
        D.set_diagonal(diag * scale)
        b = P.b * scale
        counts = []
        for prec in (False, True):
            for _ in range(2):
                x = np.zeros(n)
                ni, nr, nr0 = D.CG(b, x, 50, 1e-12, prec)
                counts.append(ni)
        assert max(counts[:2]) <= 12 and max(counts[2:]) <= 2, counts
        D.set_diagonal(diag)
        y = np.zeros(n)
        D.ComputeSPMV(P.xexact, y)
        assert np.array_equal(y, P.b)
    finally:
        D.free()


def test_symmetry_departure(binding, case32):
    """TestSymmetry.cpp:60-138 with the library's SpMV, MG and dot."""
    P, D, _, _ = case32
    n = P.levels[0].n
    rng = np.random.default_rng(17)
    x, y = rng.random(n) + 1.0, rng.random(n) + 1.0
    eps = np.finfo(float).eps
    xn, yn = binding.ComputeDotProduct(n, x, x), binding.ComputeDotProduct(n, y, y)
    z = np.zeros(n)
    D.ComputeSPMV(y, z)
    xtAy = binding.ComputeDotProduct(n, x, z)
    D.ComputeSPMV(x, z)
    ytAx = binding.ComputeDotProduct(n, y, z)
    assert abs(xtAy - ytAx) / ((xn * 52 * yn + yn * 52 * xn) * eps) <= 1.0
    D.ComputeMG(y, z)
    xtMy = binding.ComputeDotProduct(n, x, z)
    D.ComputeMG(x, z)
    ytMx = binding.ComputeDotProduct(n, y, z)
    assert abs(xtMy - ytMx) / ((xn * 52 * yn + yn * 52 * xn) * eps) <= 1.0


@pytest.mark.parametrize("cfg", [None, "1", "6", "7", "8", "9", "10"])
def test_fp32_vcycle_bitwise(oracle, binding, monkeypatch, cfg):
    """The FP32 V-cycle (autotuned, or one kernel configuration forced: rows per
    thread 1, 4 contiguous, 2 and 4 interleaved, shared-memory tiles, bulk-copy
    pipeline) is bitwise the oracle's FP32
    V-cycle on the colour order with the last colour not repeated at the turn of
    each sweep."""
    if cfg is not None:
        monkeypatch.setenv("HPCG_B200_CONFIG", cfg)
    P = oracle.generate(32, 24, 16)
    D = binding.Problem.generate(32, 24, 16)
    try:
        perms = perms_of(binding, P)
        PL = oracle.permute(P.levels, perms)
        r = np.random.default_rng(3).standard_normal(P.levels[0].n)
        x = np.zeros_like(r)
        D.ComputeMG_f32(r, x)
        if cfg is not None:
            assert D.level_config(0)["gs32"] == int(cfg)
        z = oracle.mg_f32(oracle.to_f32(PL), r[perms[0]].astype(np.float32), skip=skip_of(binding, P))
        exp = np.empty_like(r)
        exp[perms[0]] = z.astype(np.float64)
        assert np.array_equal(x, exp)
    finally:
        D.free()


def test_mixed_precision_vs_oracle(oracle, binding, case32):
    P, D, perms, PL = case32
    x = np.zeros(32 ** 3)
    ni, nr, nr0 = D.CG_mixed(P.b, x, 200, 1e-9)
    xo, nio, nro, nr0o, _ = oracle.cg_mixed(PL, P.b[perms[0]], np.zeros(32 ** 3), 200, 1e-9)
    assert abs(ni - nio) <= 1
    assert nr / nr0 <= 1e-9
    x64 = np.zeros(32 ** 3)
    D.CG(P.b, x64, 200, 1e-9, True)
    assert np.linalg.norm(x - x64) / np.linalg.norm(x64) <= 1e-7


# ---------------------------------------------------------------------------
# larger grids: size-independent properties
# ---------------------------------------------------------------------------

def test_large_grid_properties(binding):
    import torch
    n = 192
    D = binding.Problem.generate(n)
    try:
        N = n ** 3
        b = torch.zeros(N, dtype=torch.float64, device="cuda")
        D.get_rhs(b)
        ones = torch.ones(N, dtype=torch.float64, device="cuda")
        y = torch.zeros_like(ones)
        D.ComputeSPMV(ones, y)
        assert torch.equal(y, b)  # A * xexact = b exactly
        g = torch.Generator(device="cuda").manual_seed(5)
        u = torch.rand(N, dtype=torch.float64, device="cuda", generator=g)
        v = torch.rand(N, dtype=torch.float64, device="cuda", generator=g)
        Au, Av = torch.zeros_like(u), torch.zeros_like(v)
        D.ComputeSPMV(u, Au)
        D.ComputeSPMV(v, Av)
        a, c = binding.ComputeDotProduct(N, v, Au), binding.ComputeDotProduct(N, u, Av)
        assert abs(a - c) <= 1e-12 * abs(a)
        x = torch.zeros(N, dtype=torch.float64, device="cuda")
        res = []
        for k in (1, 5, 10):
            x.zero_()
            ni, nr, nr0 = D.CG(b, x, k, 0.0, True)
            res.append(nr / nr0)
        # HPCG's V-cycle (injection, 4 levels) is not size-robust: about 0.75 per
        # iteration at 128^3 in the reference, a little slower at 192^3
        assert res[0] > res[1] > res[2] and res[2] < 0.1, res
    finally:
        D.free()


# ---------------------------------------------------------------------------
# errors come back as status codes
# ---------------------------------------------------------------------------

def test_unsupported_matrix_is_rejected(oracle, binding):
    P = oracle.generate(16)
    lv = levels_of(P)
    cols = lv[0]["cols"].copy()
    cols[5 * 27 + 2] = 4000  # not a stencil neighbour of row 5
    lv[0] = dict(lv[0], cols=cols)
    with pytest.raises(binding.HpcgError) as e:
        binding.Problem.optimize(lv)
    assert e.value.status == binding.ERR_UNSUPPORTED
    lv = levels_of(P)
    f2c = lv[0]["f2c"].copy()
    f2c[3] = -1
    lv[0] = dict(lv[0], f2c=f2c)
    with pytest.raises(binding.HpcgError) as e:
        binding.Problem.optimize(lv)
    assert e.value.status == binding.ERR_ARG
    with pytest.raises(binding.HpcgError) as e:
        binding.Problem.generate(20, 20, 20, 4)  # 20 -> 10 -> 5 -> not halvable
    assert e.value.status == binding.ERR_UNSUPPORTED


def test_device_budget_gives_nomem():
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from hpcg_b200 import binding as B\n"
            "try:\n    B.Problem.generate(64)\nexcept B.HpcgError as e:\n    print('status', e.status)\n"
            "p = None\n") % os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, HPCG_B200_DEVICE_BUDGET="1000000")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "status 4" in out.stdout


def test_graph_loop_equals_stream_loop(case32):
    """The CG loop as one CUDA graph (conditional while node, the loop condition
    of CG.cpp:100 evaluated on the device) computes the same bits as the loop
    launched kernel by kernel (used when times are requested)."""
    P, D, _, _ = case32
    n = P.levels[0].n
    for max_iter, tol, prec in ((1, 0.0, True), (17, 0.0, True), (500, 1e-7, True), (30, 1e-6, False)):
        xg = np.zeros(n)
        ng = D.CG(P.b, xg, max_iter, tol, prec)
        xe = np.zeros(n)
        times = np.zeros(10)
        ne = D.CG(P.b, xe, max_iter, tol, prec, times=times)
        assert ng == ne, (max_iter, tol, prec)
        assert np.array_equal(xg, xe)
        # times[1..5] as CG.cpp:132-139 files them: dots, updates, SpMV,
        # preconditioner (or the copy z = r that replaces it, CG.cpp:105) from
        # CUDA events; one process, no allreduce (times[4] stays 0, as the
        # reference's without MPI); the parts together within the whole call
        assert times[0] > 0.0 and times[1] > 0.0 and times[2] > 0.0 and times[3] > 0.0, times
        assert times[5] > 0.0 and times[4] == 0.0
        assert times[1] + times[2] + times[3] + times[5] <= times[0], times


@pytest.mark.parametrize("cfg", ["9", "10"])
def test_cg_forced_config_vs_oracle(oracle, binding, monkeypatch, cfg):
    """CG with the phases forced to a configuration that runs its own kernel
    (shared-memory tiles, bulk-copy pipeline), r'z from the post-smoother's fused
    partials: history and x as the oracle's CG on the colour order; the graph
    loop equals the stream loop."""
    monkeypatch.setenv("HPCG_B200_CONFIG", cfg)
    P = oracle.generate(32)
    D = binding.Problem.optimize(levels_of(P))
    try:
        perms = perms_of(binding, P)
        PL = oracle.permute(P.levels, perms)
        b = P.b[perms[0]]
        for k in (1, 10, 50):
            x = np.zeros(32 ** 3)
            ni, nr, nr0 = D.CG(P.b, x, k, 0.0, True)
            assert D.level_config(0)["gs"] == int(cfg)
            xo, nio, nro, nr0o, _ = oracle.cg(PL, b, np.zeros(32 ** 3), k, 0.0, skip=skip_of(binding, P))
            assert ni == nio == k
            hist_close([nr / nr0], [nro / nr0o])
            xn = np.empty_like(xo)
            xn[perms[0]] = xo
            assert np.max(np.abs(x - xn)) <= 1e-10 * max(np.max(np.abs(xn)), 1.0)
        xg = np.zeros(32 ** 3)
        ng = D.CG(P.b, xg, 20, 0.0, True)
        xe = np.zeros(32 ** 3)
        ne = D.CG(P.b, xe, 20, 0.0, True, times=np.zeros(10))
        assert ng == ne and np.array_equal(xg, xe)
    finally:
        D.free()


@pytest.mark.parametrize("dims", [(32, 32, 32), (16, 24, 40), (24, 24, 24)])
def test_packed_columns_equal_plain_columns(binding, monkeypatch, dims):
    """The bulk-copy kernels read a level's packed column index (one record per
    128-row tile: 27 bases and the record's form, then either the diagonal
    form's sink bits, where every slot's columns across a tile are one
    diagonal, or 8-bit offsets where every tile's slot spans at most 254 rows,
    else 16-bit ones). Problems made with HPCG_B200_PACKED=8 (no diagonal
    form), =16 (16-bit offsets everywhere) and =0 (only the 32-bit columns)
    are the other three forms. Each level gets the form the numpy restatement
    of the format predicts. With the bulk-copy configurations forced, SpMV,
    SYMGS, the V-cycle and CG around the FP32 V-cycle give the same bits all
    four ways (16x24x40 and 24^3: colour blocks off the 128-row grid on some
    levels, which then take offsets, and where the slab-order SpMV keeps the
    32-bit columns). The FP64 CG forms r'z by its own dot pass on the 8- and
    16-bit forms and from the post-smoother's partials on the diagonal form and
    the 32-bit columns (whose partials follow each shape's rows per thread), so
    its history and x agree bit for bit between the two offset forms and to
    rounding otherwise. The SpMV's p'Ap partials follow its shape too (three
    consumer groups with packed records, two with 32-bit columns), so the CG
    around the FP32 V-cycle is bitwise among the packed forms and within its
    FP32-rounding bound (2^-23) of the 32-bit columns."""
    from tests.test_packed_format import packed_width
    rec = {1: 3568, 2: 7024, 3: 544}
    monkeypatch.setenv("HPCG_B200_CONFIG", "10")
    A = binding.Problem.generate(*dims)
    monkeypatch.setenv("HPCG_B200_PACKED", "8")
    E = binding.Problem.generate(*dims)
    monkeypatch.setenv("HPCG_B200_PACKED", "16")
    W = binding.Problem.generate(*dims)
    monkeypatch.setenv("HPCG_B200_PACKED", "0")
    U = binding.Problem.generate(*dims)
    try:
        for lv in range(4):
            _, pitch, _ = A.level_info(lv)
            sides = (dims[0] >> lv, dims[1] >> lv, dims[2] >> lv)
            f = packed_width(binding, *sides)
            w = packed_width(binding, *sides, diagonal=False)
            assert f in (1, 2, 3) and w in (1, 2)
            assert A.level_packed(lv) == pitch // 128 * rec[f] and A.level_pack_width(lv) == f
            assert E.level_packed(lv) == pitch // 128 * rec[w]
            assert W.level_packed(lv) == pitch // 128 * 7024
            assert U.level_packed(lv) == 0
        n = A.nrow
        b = A.get_rhs()
        rng = np.random.default_rng(7)
        v = rng.uniform(-1.0, 1.0, n)
        outs = []
        for P in (A, E, W, U):
            y = np.zeros(n)
            P.ComputeSPMV(v, y)
            xs = v.copy()
            P.ComputeSYMGS(b, xs)
            xm = np.zeros(n)
            P.ComputeMG(b, xm)
            xc = np.zeros(n)
            rc = P.CG(b, xc, 25, 0.0, True)
            xf = np.zeros(n)
            rf = P.CG_mixed(b, xf, 25, 0.0)
            assert P.level_config(0)["gs"] == 10 and P.level_config(0)["gs32"] == 10
            outs.append((y, xs, xm, xc, rc, xf, rf))
        # pairs (reference, other, FP64 CG bitwise, FP32-V-cycle CG bitwise)
        pairs = ((outs[0], outs[1], False, True), (outs[0], outs[2], False, True), (outs[1], outs[2], True, True),
                 (outs[0], outs[3], False, False))
        for ref, other, exact64, exact32 in pairs:
            for i, (a, u) in enumerate(zip(ref, other)):
                exact = exact64 if i in (3, 4) else exact32 if i in (5, 6) else True
                if exact:
                    if isinstance(a, np.ndarray):
                        assert np.array_equal(a, u), i
                    else:
                        assert a == u, i
                elif i in (3, 5):  # x of the FP64 CG / of the CG around the FP32 V-cycle
                    assert np.max(np.abs(a - u)) <= (1e-12 if i == 3 else 1e-6) * np.max(np.abs(u)), i
                else:  # (iterations, normr, normr0): the history bounds of the other CG tests
                    assert a[0] == u[0] and a[2] == u[2], i
                    hist_close([a[1] / a[2]], [u[1] / u[2]], rel=1e-10 if i == 4 else 2.0 ** -23)
    finally:
        A.free()
        E.free()
        W.free()
        U.free()


def test_bounded_wait_gives_up_and_context_survives(oracle, binding, case16):
    """The device-side wait of the bulk-copy phases ends by itself: waiting on an
    mbarrier that nothing completes returns HPCG_B200_ERR_TIMEOUT after the
    limit, and the same context then runs the V-cycle bit for bit."""
    import time
    t0 = time.perf_counter()
    st = binding.wait_selftest(0.25)
    dt = time.perf_counter() - t0
    assert st == binding.ERR_TIMEOUT
    assert 0.2 <= dt < 30.0
    assert "gave up" in binding.last_error()
    P, D, perms, PL = case16
    r = np.random.default_rng(11).standard_normal(16 ** 3)
    z = np.zeros_like(r)
    D.ComputeMG(r, z)
    exp = np.empty_like(z)
    exp[perms[0]] = oracle.mg(PL, r[perms[0]], skip=skip_of(binding, P))
    assert np.array_equal(z, exp)
    with pytest.raises(binding.HpcgError):
        binding._check(binding.lib().hpcg_b200_wait_selftest(0, 5.0), "wait_selftest")


@pytest.mark.parametrize("packed", ["", "0"])
def test_stream_probe_reads_the_matrix_only(binding, monkeypatch, packed):
    """hpcg_b200_stream_probe streams every 128-row tile of a level (values
    and column index, in the level's column form) through the phases' copy
    pipeline and changes nothing: the bytes it reports are the tiles' bytes,
    and a V-cycle after it gives the same bits as before."""
    if packed:
        monkeypatch.setenv("HPCG_B200_PACKED", packed)
    D = binding.Problem.generate(64, 32, 48)
    try:
        r = np.random.default_rng(5).standard_normal(D.nrow)
        z0 = np.zeros_like(r)
        D.ComputeMG(r, z0)
        for level in range(4):
            n, pitch, _ = D.level_info(level)
            ms, nb = D.stream_probe(level)
            form = D.level_pack_width(level)
            rec = {0: 27 * 128 * 4, 1: 28 * 4 + 27 * 128, 2: 28 * 4 + 27 * 256, 3: 28 * 4 + 27 * 16}[form]
            assert nb == -(-n // 128) * (27 * 128 * 8 + rec), (level, form, nb)
            assert ms > 0.0
        z1 = np.zeros_like(r)
        D.ComputeMG(r, z1)
        assert np.array_equal(z0, z1)
    finally:
        D.free()
    with pytest.raises(binding.HpcgError):
        binding._check(binding.lib().hpcg_b200_stream_probe(None, 0, None, None), "stream_probe")


def test_stream_vcycle_follows_coarse_value_changes(oracle, binding):
    """The loops that launch kernel by kernel run the V-cycle below level 0 as
    one captured graph. After set_values on a coarse level (which rebuilds that
    level's FP32 copy at a new address), the FP64 and FP32 V-cycles equal those
    of a problem built with the new values from the start."""
    P = oracle.generate(32)
    lv = levels_of(P)
    lv2 = [dict(d) for d in lv]
    lv2[1]["vals"] = lv[1]["vals"] * 1.5
    D1 = binding.Problem.optimize(lv)
    D2 = binding.Problem.optimize(lv2)
    try:
        n = P.levels[0].n
        r = np.random.default_rng(17).standard_normal(n)
        z = np.zeros(n)
        D1.ComputeMG(r, z)
        D1.ComputeMG_f32(r, z)  # both coarse graphs captured on the old values
        e = D2.export_level(1)
        m = e["n"]
        v27 = np.zeros((m, 27))
        v27[e["new2old"]] = e["vals"][:, :m].T
        D1.set_values(1, v27)
        for f in (lambda D, x: D.ComputeMG(r, x), lambda D, x: D.ComputeMG_f32(r, x)):
            a, b = np.zeros(n), np.zeros(n)
            f(D1, a)
            f(D2, b)
            assert np.array_equal(a, b)
    finally:
        D1.free()
        D2.free()
