"""Host side of the run over several ranks, no GPU needed.

* The process grid equals the reference's ComputeOptimalShapeXYZ for 1..400 ranks.
* The halo plan (neighbours, counts, rows sent, external numbering) equals the
  one the reference's own SetupHalo_ref builds in its MPI branch, run here as
  threads over the MPI stand-in of oracle/mpi_shim, on every rank and level.
* Plans pair up across ranks: what rank a sends to b is, entry for entry, what
  b numbers as its externals from a, also when each rank computes its plan in
  its own process (world size 2 over gloo).
"""
import os
import socket

import numpy as np
import pytest

DECOMPS = [(2, 1, 1, 16, 16, 16), (1, 1, 2, 16, 16, 16), (2, 2, 2, 8, 8, 8), (3, 2, 1, 8, 16, 8),
           (3, 3, 3, 8, 8, 8), (2, 3, 4, 8, 8, 16)]


def _ref_ranks(oracle):
    if not oracle.have_reference_ranks():
        pytest.skip("oracle/_ref/libhpcg_ref_mpi.so not built (needs the reference sources)")
    return oracle.ReferenceRanks


def test_process_grid_matches_reference(oracle, binding):
    R = _ref_ranks(oracle)
    for n in range(1, 401):
        assert binding.process_grid(n) == R.optimal_shape(n), n


@pytest.mark.parametrize("decomp", DECOMPS)
def test_halo_plan_matches_setup_halo(oracle, binding, decomp):
    R = _ref_ranks(oracle)
    px, py, pz, nx, ny, nz = decomp
    ref = R(px, py, pz, nx, ny, nz)
    try:
        for rank in range(px * py * pz):
            for lev in range(4):
                d = (nx >> lev, ny >> lev, nz >> lev)
                e = ref.export(rank, lev)
                p = binding.halo_plan(*d, px, py, pz, rank)
                assert np.array_equal(e["neighbors"], p["neighbors"]), (rank, lev)
                assert np.array_equal(e["recv_len"], p["counts"]), (rank, lev)
                assert np.array_equal(e["send_len"], p["counts"]), (rank, lev)
                assert np.array_equal(e["send_rows"], p["send_rows"]), (rank, lev)
                assert np.array_equal(e["ext_global"], p["ext_global"]), (rank, lev)
                assert e["ncol"] - e["n"] == p["counts"].sum()
    finally:
        ref.close()


def _global_rows(nx, ny, nz, px, py, pz, rank, local_rows):
    ipz, rem = divmod(rank, px * py)
    ipy, ipx = divmod(rem, px)
    x = local_rows % nx + ipx * nx
    y = (local_rows // nx) % ny + ipy * ny
    z = local_rows // (nx * ny) + ipz * nz
    return (z * (py * ny) + y) * (px * nx) + x


def _sent_to(binding, decomp, rank):
    """{neighbour: global rows rank sends it}, {neighbour: global rows rank expects from it}."""
    px, py, pz, nx, ny, nz = decomp
    p = binding.halo_plan(nx, ny, nz, px, py, pz, rank)
    off = np.concatenate([[0], np.cumsum(p["counts"])])
    g = _global_rows(nx, ny, nz, px, py, pz, rank, p["send_rows"].astype(np.int64))
    send = {int(b): g[off[i]:off[i + 1]] for i, b in enumerate(p["neighbors"])}
    recv = {int(b): p["ext_global"][off[i]:off[i + 1]] for i, b in enumerate(p["neighbors"])}
    return send, recv


@pytest.mark.parametrize("decomp", DECOMPS + [(4, 4, 2, 8, 8, 8)])
def test_halo_plans_pair_up(binding, decomp):
    px, py, pz = decomp[:3]
    plans = [_sent_to(binding, decomp, r) for r in range(px * py * pz)]
    for a, (send_a, _) in enumerate(plans):
        for b, rows in send_a.items():
            assert np.array_equal(rows, plans[b][1][a]), (a, b)


def test_rank_arguments_rejected(binding):
    with pytest.raises(binding.HpcgError):
        binding.halo_plan(8, 8, 8, 2, 1, 1, 2)  # rank outside the grid
    with pytest.raises(binding.HpcgError):
        binding.halo_plan(8, 8, 8, 0, 1, 1, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _gloo_rank(rank, world, port, decomp, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from hpcg_b200 import binding as B
        send, recv = _sent_to(B, decomp, rank)
        gathered = [None] * world
        dist.all_gather_object(gathered, {k: v.tolist() for k, v in send.items()})
        ok = all(np.array_equal(np.array(gathered[b][rank]), recv[b]) for b in recv)
        out.put((rank, ok, sorted(recv)))
    finally:
        dist.destroy_process_group()


def test_halo_plan_pairs_across_processes():
    """Each rank builds its plan in its own process; the sends gathered over gloo
    match every receiver's external numbering."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    decomp = (2, 1, 1, 16, 8, 8)
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, decomp, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == [(0, True, [1]), (1, True, [0])]


def test_dropin_mpi_branch_compiles():
    """The drop-in's MPI branch (generate_rank + NCCL communicator + shard calls)
    type-checks against the MPI stand-in's declarations and the reference headers."""
    import subprocess
    import __graft_entry__
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    ref = __graft_entry__._reference_tree()
    if ref is None:
        pytest.skip("reference sources not available here")
    r = subprocess.run(["make", "-s", "-C", os.path.join(root, "oracle"), "dropin-mpi-syntax", f"REF={ref}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
