"""Host-side logic that needs no GPU: the C ABI loads and exports every declared
symbol, argument and handle errors come back as status codes, the colour order
is a valid 8-colouring with the injected points last, and the work models
match the reference's numbers."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hpcg_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(hpcg_b200_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(binding):
    lib = binding.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(binding.EXPORTS)
    out = subprocess.run(["nm", "-D", "--defined-only", binding.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (hpcg_b200_\w+)", out))
    assert set(syms) <= exported


def test_build_targets_sm100a():
    mk = open(os.path.join(ROOT, "hpcg_b200", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk and "-fmad=false" in mk


def test_handle_and_argument_errors(binding):
    import ctypes as C
    lib = binding.lib()
    d = C.c_double(0)
    assert lib.hpcg_b200_spmv(None, None, None) == binding.ERR_HANDLE
    assert lib.hpcg_b200_symgs(None, None, None) == binding.ERR_HANDLE
    assert lib.hpcg_b200_mg(None, None, None) == binding.ERR_HANDLE
    assert lib.hpcg_b200_free(None) == binding.ERR_HANDLE
    assert lib.hpcg_b200_memory_use(None) == 0.0
    assert lib.hpcg_b200_optimize(None, 4, 0, None) == binding.ERR_ARG
    assert lib.hpcg_b200_dot(-1, None, None, C.byref(d)) == binding.ERR_ARG
    assert lib.hpcg_b200_waxpby(4, 1.0, None, 1.0, None, None) == binding.ERR_ARG
    assert lib.hpcg_b200_colour_permutation(0, 4, 4, None, None) == binding.ERR_ARG
    # a corrupted handle: not a problem object
    junk = (C.c_uint64 * 64)()
    assert lib.hpcg_b200_spmv(C.cast(junk, C.c_void_p), None, None) == binding.ERR_HANDLE
    assert lib.hpcg_b200_set_symgs_mode(C.cast(junk, C.c_void_p), 0) == binding.ERR_HANDLE
    b = C.c_int64(-1)
    assert lib.hpcg_b200_level_packed(None, 0, C.byref(b)) == binding.ERR_HANDLE
    assert lib.hpcg_b200_level_packed(C.cast(junk, C.c_void_p), 0, C.byref(b)) == binding.ERR_HANDLE
    assert b.value == -1  # nothing written on an error


def test_no_gpu_is_a_clean_error(binding):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(binding.HpcgError) as e:
        binding.Problem.generate(16)
    assert e.value.status == binding.ERR_CUDA


@pytest.mark.parametrize("dims", [(16, 16, 16), (32, 16, 24), (24, 24, 24), (3, 3, 3), (2, 4, 6), (1, 1, 1)])
def test_colour_order_is_a_valid_colouring(binding, oracle, dims):
    nx, ny, nz = dims
    n2o, starts = binding.colour_permutation(nx, ny, nz)
    n = nx * ny * nz
    assert sorted(n2o.tolist()) == list(range(n))
    assert starts[0] == 0 and starts[8] == n and np.all(np.diff(starts) >= 0)
    col = oracle.parity_colour(nx, ny, nz)
    colour_of_row = np.empty(n, np.int32)
    for s in range(8):
        blk = n2o[starts[s]:starts[s + 1]]
        assert len(set(col[blk].tolist())) <= 1
        colour_of_row[blk] = s
        # natural order inside a colour block
        assert np.all(np.diff(blk) > 0)
    # no two stencil neighbours share a colour
    L = oracle.generate_level(nx, ny, nz)
    cols, _ = L.dense_rows()
    for i in range(n):
        nb = cols[i, : L.nnz[i]]
        nb = nb[nb != i]
        assert np.all(colour_of_row[nb] != colour_of_row[i])
    # the injected points (all coordinates even) are swept last
    if nx % 2 == 0 and ny % 2 == 0 and nz % 2 == 0:
        last = n2o[starts[7]:starts[8]]
        iz, rem = np.divmod(last, nx * ny)
        iy, ix = np.divmod(rem, nx)
        assert np.all(ix % 2 == 0) and np.all(iy % 2 == 0) and np.all(iz % 2 == 0)


def test_colour_order_matches_oracle_sweep(binding, oracle):
    n2o, _ = binding.colour_permutation(16, 16, 16)
    assert np.array_equal(n2o, oracle.colour_new2old(16, 16, 16, [7, 6, 3, 5, 4, 1, 2, 0]))


def test_colour_order_convergence(binding, oracle):
    """CG on the colour-ordered system reaches the natural-order 50-iteration
    residual within a few extra iterations (HPCG charges extra iterations in the
    rating, ReportResults.cpp:99)."""
    P = oracle.generate(32)
    _, _, nr, nr0, _ = oracle.cg(P.levels, P.b, P.x, 50, 0.0)
    ref_tol = nr / nr0
    perms = [binding.colour_permutation(L.nx, L.ny, L.nz)[0] for L in P.levels]
    PL = oracle.permute(P.levels, perms)
    _, ni, nr, nr0, _ = oracle.cg(PL, P.b[perms[0]], np.zeros(32 ** 3), 500, ref_tol)
    assert nr / nr0 <= ref_tol
    assert ni <= 60


def test_flop_and_byte_models(oracle):
    from hpcg_b200 import metrics
    import json
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "golden_32.json")))
    assert metrics.hpcg_flops(32, 32, 32, 50) == g["flops_50"]
    assert [z for _, z in metrics.level_sizes(32, 32, 32)] == g["nnz_per_level"]
    assert metrics.level_sizes(512, 512, 512)[0][1] == 3609741304
    assert abs(metrics.compulsory_bytes(512, 512, 512) / 1e9 - 282.1) < 0.1
    per_iter = metrics.hpcg_flops(512, 512, 512, 51) - metrics.hpcg_flops(512, 512, 512, 50)
    assert abs(per_iter / 5.0162e10 - 1) < 5e-3  # 5.0007e10 by the exact formula


def test_iteration_byte_model():
    """metrics.iteration_bytes, the floor the library's kernels move per CG
    iteration: the index width enters only through the bulk-copy kernels'
    records (27.875 / 54.875 / 108 B per row; 4.25 for the diagonal form),
    an r'z pass only where the post-smoother does not fuse it, the FP32 V-cycle halves the
    V-cycle's value and vector bytes but not the FP64 SpMV and CG vectors."""
    from hpcg_b200 import metrics
    assert metrics.index_bytes_per_row(1) == 27.875 and metrics.index_bytes_per_row(2) == 54.875
    assert metrics.index_bytes_per_row(0) == 108
    b = {w: metrics.iteration_bytes(512, 512, 512, 8, (w,) * 4) for w in (0, 1, 2)}
    assert b[1] < b[2] < b[0]
    assert abs(b[2] / 1e9 - 232.97) < 0.01  # 16-bit offsets, every level
    assert abs(b[1] / 1e9 - 217.46) < 0.01  # 8-bit offsets, every level
    # the diagonal form's post-smoother accumulates r'z: no 16 B/row pass of its own
    d = metrics.iteration_bytes(512, 512, 512, 8, (3,) * 4)
    assert abs(d / 1e9 - 201.74) < 0.01
    assert metrics.iteration_bytes(512, 512, 512, 8, (3,) * 4, rtz_fused=False) - d == 16 * 512 ** 3
    t, parts = metrics.iteration_bytes(512, 512, 512, 4, (1,) * 4, parts=True)
    assert abs(sum(parts.values()) * 1e9 - t) < 1.0
    assert parts["spmv"] == metrics.spmv_bytes(512 ** 3, 8, 1) / 1e9 and parts["vectors"] == 96 * 512 ** 3 / 1e9
    assert 0.66 < t / b[1] < 0.67


def test_gpu_launch_count_model():
    import bench
    # 16 launches per symmetric sweep would double count; the model is 15 per sweep.
    # Per iteration besides the V-cycle: r'z finalize (partials from the
    # post-smoother), p update (with the previous x update), SpMV + finalize,
    # r update + finalize = 6, which makes the 117 launches per iteration of the
    # 512^3 launch list; one x update after the loop.
    assert bench.gpu_launches_per_set(1) == (32 * 3 + 15) + 6 - 1 + 3 + 3 + 1
    assert bench.gpu_launches_per_set(2) - bench.gpu_launches_per_set(1) == 117
    # level 0 on the packed bulk-copy phases: r'z as its own dot kernel
    assert bench.gpu_launches_per_set(2, rtz_pass=True) - bench.gpu_launches_per_set(1, rtz_pass=True) == 118
