"""The changed forms pinned directly to the oracle (needs a B200), not only to
the GPU's own single-system path.

Each form runs on the library's colour order, so the oracle runs the reference
routines on the colour-permuted hierarchy with the last colour of each sweep not
repeated at the turn (ora_mg_skip / ora_mg_f32_skip / ora_cg_skip /
ora_cg_mixed_skip, restating ComputeMG_ref.cpp:39-63, ComputeSYMGS_ref.cpp:54-103
and CG_ref.cpp:58-144).

* FP64 flexible CG around the FP32 V-cycle (hpcg_b200_cg_mixed), against the
  oracle's flexible CG on the same FP32 V-cycle. The first iteration's
  V-cycle input is float(b) on both sides, so its scaled residual agrees
  within the CG history bound of the other tests, |d| <= 1e-10 * max(r, 1e-9).
  After it, the FP64 residuals differ in their last bits (dot products summed
  in another order) and a last-bit difference can flip the rounding of r to
  FP32 at the V-cycle's input: later iterations agree within FP32 rounding,
  |d| <= 2^-23 * max(r, 1e-9), checked at every iteration count whose scaled
  residual is still at or above 1e-5 (measured up to 1.5e-8 relative there).
  The difference then grows by about 1.75x per iteration (3.5e-4 relative at
  iteration 30, scaled residual 2.4e-12): two runs of the form whose FP32
  roundings of r differ follow trajectories that separate geometrically while
  both converge. So beyond that point only the solutions are compared: x after
  30 iterations within 1e-6 of max|x|.
* Several right-hand sides (hpcg_b200_mg_multi / _cg_multi): each system's
  V-cycle bit for bit the oracle's V-cycle, each system's CG history within
  the same bound of the oracle's CG_ref, on U[-1,1] right-hand sides.
* Batched problems (hpcg_b200_batch_cg_mixed): each problem's history against
  the oracle's flexible CG at fixed iteration counts, with the mixed form's
  two bounds.

Dot products reduce in a fixed tree on the GPU and serially in the oracle, so
CG histories agree to rounding, not bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(oracle, binding, dims):
    from tests.test_gpu_parity import perms_of, skip_of
    P = oracle.generate(*dims)
    perms = perms_of(binding, P)
    PL = oracle.permute(P.levels, perms)
    return P, perms, PL, skip_of(binding, P)


def _natural(v, perm):
    out = np.empty_like(v)
    out[perm] = v
    return out


def _hist_close(a, b, rel=1e-10):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    bound = rel * np.maximum(np.abs(b), 1e-9)
    assert np.all(np.abs(a - b) <= bound), (a, b)


FP32_ROUNDING = 2.0 ** -23  # a flipped FP32 rounding of r, relative


def _mixed_close(k, ours, hist):
    _hist_close([ours], [hist[k] / hist[0]], rel=1e-10 if k == 1 else FP32_ROUNDING)


def _uniform(n, seed):
    return np.random.Generator(np.random.PCG64(seed)).uniform(-1.0, 1.0, n)


@pytest.mark.parametrize("dims,rhs", [((32, 32, 32), "hpcg"), ((32, 32, 32), "uniform"),
                                      ((24, 16, 40), "uniform")])
def test_mixed_cg_history_vs_oracle(oracle, binding, dims, rhs):
    P, perms, PL, skip = _setup(oracle, binding, dims)
    n = P.levels[0].n
    b = P.b if rhs == "hpcg" else _uniform(n, 0x48504347)
    K = 30
    xo, nio, _, _, hist = oracle.cg_mixed(PL, b[perms[0]], np.zeros(n), K, 0.0, skip=skip)
    assert nio == K
    checked = [k for k in (1, 2, 3, 5, 8, 10, 12, 14) if hist[k] / hist[0] >= 1e-5]
    assert len(checked) >= 5
    D = binding.Problem.generate(*dims)
    try:
        for k in checked:
            x = np.zeros(n)
            ni, nr, nr0 = D.CG_mixed(b, x, k, 0.0)
            assert ni == k
            assert abs(nr0 - hist[0]) <= 1e-13 * hist[0]
            _mixed_close(k, nr / nr0, hist)
        x = np.zeros(n)
        assert D.CG_mixed(b, x, K, 0.0)[0] == K
        xn = _natural(xo, perms[0])
        assert np.max(np.abs(x - xn)) <= 1e-6 * max(np.max(np.abs(xn)), 1.0)
    finally:
        D.free()


@pytest.mark.parametrize("dims", [(32, 32, 32), (24, 16, 40)])
def test_multi_rhs_vs_oracle(oracle, binding, dims):
    P, perms, PL, skip = _setup(oracle, binding, dims)
    n = P.levels[0].n
    K = 8
    r = np.stack([_uniform(n, 100 + j) for j in range(K)])
    D = binding.Problem.generate(*dims)
    try:
        z = np.zeros((K, n))
        D.ComputeMG_multi(r, z)
        for j in range(K):
            zo = oracle.mg(PL, r[j][perms[0]], skip=skip)
            assert np.array_equal(z[j], _natural(zo, perms[0])), j
        iters = 12
        hists = [oracle.cg(PL, r[j][perms[0]], np.zeros(n), iters, 0.0, skip=skip)[4] for j in range(K)]
        for k in (1, 4, iters):
            x = np.zeros((K, n))
            ni, nr, nr0 = D.CG_multi(r, x, k, 0.0)
            for j in range(K):
                assert ni[j] == k
                assert abs(nr0[j] - hists[j][0]) <= 1e-13 * hists[j][0]
                _hist_close([nr[j] / nr0[j]], [hists[j][k] / hists[j][0]])
    finally:
        D.free()


def test_batched_vs_oracle(oracle, binding):
    dims = [(16, 32, 48), (32, 16, 16), (16, 16, 16)]
    setups = [_setup(oracle, binding, d) for d in dims]
    bs = [_uniform(s[0].levels[0].n, 7 + i) for i, s in enumerate(setups)]
    bs[1] = setups[1][0].b.copy()
    K = 10
    hists = []
    for (P, perms, PL, skip), b in zip(setups, bs):
        n = P.levels[0].n
        _, nio, _, _, h = oracle.cg_mixed(PL, b[perms[0]], np.zeros(n), K, 0.0, skip=skip)
        assert nio == K
        hists.append(h)
    B = binding.Batch(dims)
    try:
        for k in (1, 4, K):
            xs = [np.zeros(s[0].levels[0].n) for s in setups]
            ni, nr, nr0 = B.CG_mixed(bs, xs, k, 0.0)
            for i, h in enumerate(hists):
                assert ni[i] == k
                assert abs(nr0[i] - h[0]) <= 1e-13 * h[0]
                if h[k] / h[0] >= 1e-5:  # see the module docstring
                    _mixed_close(k, nr[i] / nr0[i], h)
    finally:
        B.free()
