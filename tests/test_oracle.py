"""The oracle pinned: the C restatement against the golden vectors produced by
the HPCG 3.1 reference itself, and (where oracle/_ref was built) against the
reference routines directly. CPU only."""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def g16():
    return np.load(os.path.join(GOLD, "golden_16.npz"))


@pytest.fixture(scope="module")
def g32():
    with open(os.path.join(GOLD, "golden_32.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def p16(oracle):
    return oracle.generate(16)


def test_generate_matches_golden(oracle, p16, g16):
    assert np.array_equal(p16.b, g16["b"])
    assert np.array_equal(p16.xexact, g16["xexact"])
    assert np.all(p16.x == 0.0)


def test_kernels_bitwise_vs_golden(oracle, p16, g16):
    xs = g16["x_seed"]
    A = p16.levels[0]
    assert np.array_equal(oracle.spmv(A, xs), g16["spmv"])
    assert np.array_equal(oracle.symgs(A, p16.b, xs), g16["symgs"])
    assert np.array_equal(oracle.mg(p16.levels, xs), g16["mg"])


def test_cg_history_vs_golden(oracle, p16, g16):
    _, ni, nr, nr0, hist = oracle.cg(p16.levels, p16.b, p16.x, 20, 0.0)
    assert ni == 20
    assert nr0 == g16["normr0"]
    assert np.array_equal(hist[1:] / hist[0], g16["cg_hist"])
    x10 = oracle.cg(p16.levels, p16.b, p16.x, 10, 0.0)[0]
    assert np.array_equal(x10, g16["cg_x10"])


def test_permuted_cg_matches_reference_on_permuted_system(oracle, binding, p16, g16):
    """The oracle's renumbering reproduces CG_ref run by the reference on its own
    structures renumbered the same way (oracle/ref_bridge.cpp ref_permute)."""
    perms = [binding.colour_permutation(L.nx, L.ny, L.nz)[0] for L in p16.levels]
    assert np.array_equal(perms[0], g16["perm0"])
    PL = oracle.permute(p16.levels, perms)
    _, ni, nr, nr0, hist = oracle.cg(PL, p16.b[perms[0]], np.zeros(16 ** 3), 20, 0.0)
    assert np.array_equal(hist[1:] / hist[0], g16["cg_hist_perm"])


def test_known_answers_32(oracle, g32):
    """The 32^3 pins: initial residual 722.003, scaled residual 0.183273 after 1
    iteration ... 1.02983e-20 after 50 (reference run, serial, strict IEEE)."""
    P = oracle.generate(32)
    assert [L.total_nnz for L in P.levels] == g32["nnz_per_level"]
    _, ni, nr, nr0, hist = oracle.cg(P.levels, P.b, P.x, 50, 0.0)
    assert nr0 == pytest.approx(722.003, rel=1e-6)
    assert nr0 == g32["normr0"]
    for k, v in g32["scaled_residual"].items():
        assert hist[int(k)] / hist[0] == v
    assert hist[1] / hist[0] == pytest.approx(0.183273, rel=1e-5)
    assert hist[23] / hist[0] == pytest.approx(1.05496e-09, rel=1e-5)


def test_vector_routines(oracle):
    rng = np.random.default_rng(3)
    x, y = rng.standard_normal(1000), rng.standard_normal(1000)
    assert oracle.dot(x, y) == sum(float(a) * float(b) for a, b in zip(x, y)) or \
        abs(oracle.dot(x, y) - float(np.dot(x, y))) < 1e-12
    w = oracle.waxpby(2.5, x, -0.5, y)
    assert np.array_equal(w, 2.5 * x + -0.5 * y)
    assert np.array_equal(oracle.waxpby(1.0, x, 3.0, y), x + 3.0 * y)
    assert oracle.residual(x, y) == np.max(np.abs(x - y))


@pytest.mark.parametrize("dims", [(16, 24, 32), (24, 24, 24), (16, 16, 16)])
def test_oracle_against_reference_build(oracle, dims):
    """Non-cubic grids and an odd coarsest level (24 -> 3): the restatement and
    the reference agree bit for bit on every routine."""
    if not oracle.have_reference():
        pytest.skip("oracle/_ref/libhpcg_ref.so not built (reference tree absent at build time)")
    P = oracle.generate(*dims)
    R = oracle.Reference(*dims)
    for l, L in enumerate(R.levels()):
        M = P.levels[l]
        assert np.array_equal(M.nnz, L.nnz) and np.array_equal(M.cols, L.cols)
        assert np.array_equal(M.vals, L.vals) and np.array_equal(M.diag, L.diag)
        if l < 3:
            assert np.array_equal(M.f2c, L.f2c)
    xs = np.random.default_rng(1).random(P.levels[0].n)
    assert np.array_equal(oracle.spmv(P.levels[0], xs), R.spmv(xs))
    assert np.array_equal(oracle.symgs(P.levels[0], P.b, xs), R.symgs(P.b, xs))
    assert np.array_equal(oracle.mg(P.levels, xs), R.mg(xs))
    xo = oracle.cg(P.levels, P.b, P.x, 15, 0.0)[0]
    xr = R.cg(15, 0.0)[0]
    assert np.array_equal(xo, xr)
    assert R.test_cg()["count_fail"] == 0


def test_mixed_precision_oracle_converges(oracle):
    """FP32 V-cycle in flexible FP64 CG reaches 1e-9 at 32^3 within a few more
    iterations than FP64."""
    P = oracle.generate(32)
    _, ni64, nr, nr0, _ = oracle.cg(P.levels, P.b, P.x, 200, 1e-9)
    _, ni32, nr32, nr032, _ = oracle.cg_mixed(P.levels, P.b, P.x, 200, 1e-9)
    assert nr / nr0 <= 1e-9 and nr32 / nr032 <= 1e-9
    assert ni32 <= ni64 + 3
