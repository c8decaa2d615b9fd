"""The wavefront sweeps (wave.cuh, hpcg_b200_level_wavefront): each FP64 sweep
that starts from a nonzero x as one cooperative launch, phase j two z pairs
behind phase j - 1. Every row reads the same neighbour values as in the
phase-by-phase sweep, so the V-cycle is bitwise the same (and bitwise the
oracle's colour-order ora_mg with the turn colour skipped). The CG's r'z
partials are summed in a different grouping (one partial per block of the
sweep instead of one per block of each phase), so CG histories are compared
with the oracle's at the usual 1e-10 on the scaled residual.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# grid shapes whose levels 0 and 1 (and for the first, level 2) cut into
# whole 128-row tiles per colour and z pair, the coarse ones not
SHAPES = [(64, 64, 32), (64, 32, 48), (32, 32, 64)]


def config_with_wave(binding, dims, wf):
    """A pinned HPCG_B200_LEVEL_CONFIG for a problem of these sides: the tuned
    choices of one problem, with the wavefront field set to wf on every level."""
    T = binding.Problem.generate(*dims)
    try:
        r = np.zeros(T.nrow)
        T.ComputeMG(r, r.copy())
        parts = T.level_config_string().split(";")
    finally:
        T.free()
    return ";".join(",".join(p.split(",")[:6] + [str(wf)]) for p in parts)


def eligible(nx, ny, nz):
    return nx % 2 == 0 and ny % 2 == 0 and nz % 2 == 0 and (nx // 2) * (ny // 2) % 128 == 0


@pytest.mark.parametrize("dims", SHAPES)
def test_wave_vcycle_bitwise_vs_phases_and_oracle(oracle, binding, monkeypatch, dims):
    from test_gpu_parity import levels_of, perms_of, skip_of
    r = np.random.default_rng(sum(dims)).standard_normal(int(np.prod(dims)))
    out = {}
    for wf in (0, 1):
        monkeypatch.setenv("HPCG_B200_LEVEL_CONFIG", config_with_wave(binding, dims, wf))
        D = binding.Problem.generate(*dims)
        try:
            z = np.zeros_like(r)
            D.ComputeMG(r, z)
            out[wf] = z
            for l in range(D.nlevels):
                nx, ny, nz = dims[0] >> l, dims[1] >> l, dims[2] >> l
                assert D.level_wavefront(l) == (wf if eligible(nx, ny, nz) else 0), l
            if wf:
                x1 = np.random.default_rng(7).standard_normal(r.size)
                x0 = x1.copy()
                D.ComputeSYMGS(r, x1)  # one symmetric step from nonzero x: both sweeps are wavefronts
                monkeypatch.setenv("HPCG_B200_LEVEL_CONFIG", config_with_wave(binding, dims, 0))
                E = binding.Problem.generate(*dims)
                try:
                    E.ComputeSYMGS(r, x0)
                finally:
                    E.free()
                assert np.array_equal(x1, x0)
        finally:
            D.free()
    assert np.array_equal(out[0], out[1])
    P = oracle.generate(*dims)
    perms = perms_of(binding, P)
    PL = oracle.permute(P.levels, perms)
    p0 = perms[0]
    exp = np.empty_like(r)
    exp[p0] = oracle.mg(PL, r[p0], skip=skip_of(binding, P))
    assert np.array_equal(out[1], exp)


def test_wave_cg_history_vs_oracle(oracle, binding, monkeypatch):
    from test_gpu_parity import hist_close, perms_of, skip_of
    dims = (64, 64, 32)
    monkeypatch.setenv("HPCG_B200_LEVEL_CONFIG", config_with_wave(binding, dims, 1))
    D = binding.Problem.generate(*dims)
    try:
        P = oracle.generate(*dims)
        perms = perms_of(binding, P)
        PL = oracle.permute(P.levels, perms)
        n = int(np.prod(dims))
        for k in (1, 5, 20):
            x = np.zeros(n)
            ni, nr, nr0 = D.CG(P.b, x, k, 0.0, True)
            xo, nio, nro, nr0o, _ = oracle.cg(PL, P.b[perms[0]], np.zeros(n), k, 0.0, skip=skip_of(binding, P))
            assert ni == nio == k
            assert abs(nr0 - nr0o) <= 1e-13 * nr0o
            hist_close([nr / nr0], [nro / nr0o])
            xn = np.empty_like(xo)
            xn[perms[0]] = xo
            assert np.max(np.abs(x - xn)) <= 1e-10 * max(np.max(np.abs(xn)), 1.0)
        assert D.level_wavefront(0) == 1  # (levels are configured on first use)
    finally:
        D.free()


def test_wave_dependency_wait_gives_up_and_context_survives(binding, monkeypatch):
    """The sweep's dependency wait ends by itself: a unit that waits for its
    own tiles makes every block's wait run out after the limit, the call returns
    HPCG_B200_ERR_TIMEOUT with the wavefront message, and the same problem then
    runs a V-cycle with wavefront sweeps bit for bit as before."""
    dims = (64, 64, 32)
    monkeypatch.setenv("HPCG_B200_LEVEL_CONFIG", config_with_wave(binding, dims, 1))
    D = binding.Problem.generate(*dims)
    try:
        r = np.random.default_rng(3).standard_normal(D.nrow)
        z0 = np.zeros_like(r)
        D.ComputeMG(r, z0)
        t0 = time.perf_counter()
        st = D.wave_wait_selftest(0.25)
        dt = time.perf_counter() - t0
        assert st == binding.ERR_TIMEOUT
        assert 0.2 <= dt < 30.0
        assert "wavefront" in binding.last_error()
        z1 = np.zeros_like(r)
        D.ComputeMG(r, z1)
        assert np.array_equal(z0, z1)
    finally:
        D.free()
