"""HPCG work models used to turn timings into GFLOP/s and GB/s.

* ``hpcg_flops`` -- the reference's FLOP model, src/ReportResults.cpp:75-99.
* ``hpcg_model_bytes`` -- the reference's read+write model, src/ReportResults.cpp:101-136.
* ``compulsory_bytes`` -- the bytes one CG iteration must move between HBM and
  the SMs when each kernel streams its matrix rows once (the roofline numerator
  of the whole iteration).
* ``gs_phase_bytes`` -- the algorithmic bytes of one Gauss-Seidel colour phase
  (the roofline numerator of the dominant kernel).

All sizes follow the generated problem: level l of an (nx, ny, nz) grid has
(nx>>l)(ny>>l)(nz>>l) rows and (3nx_l-2)(3ny_l-2)(3nz_l-2) nonzeros.
"""
from __future__ import annotations

SLOTS = 27


def level_sizes(nx, ny, nz, nlevels=4):
    """[(rows, nnz)] per level."""
    out = []
    for l in range(nlevels):
        a, b, c = nx >> l, ny >> l, nz >> l
        out.append((a * b * c, (3 * a - 2) * (3 * b - 2) * (3 * c - 2)))
    return out


def hpcg_flops(nx, ny, nz, iters, sets=1, nlevels=4):
    """ReportResults.cpp:75-98: fnops for `sets` CG sets of `iters` iterations
    (one preamble per set), 1 pre- and 1 post-smoothing step per level."""
    lv = level_sizes(nx, ny, nz, nlevels)
    nrow, nnz = lv[0]
    fniters = sets * iters
    f = (3.0 * fniters + sets) * 2.0 * nrow        # ddot
    f += (3.0 * fniters + sets) * 2.0 * nrow       # waxpby
    f += (fniters + sets) * 2.0 * nnz              # spmv
    for l in range(nlevels - 1):
        f += fniters * (4.0 + 2.0 + 4.0) * lv[l][1]  # pre-smoother, fine residual, post-smoother
    f += fniters * 4.0 * lv[-1][1]                 # coarsest SYMGS
    return f


def hpcg_model_bytes(nx, ny, nz, iters, sets=1, nlevels=4):
    """ReportResults.cpp:101-136: reads + writes of the reference's byte model."""
    lv = level_sizes(nx, ny, nz, nlevels)
    nrow, nnz = lv[0]
    d, i = 8.0, 4.0
    fniters = sets * iters
    rd = (3.0 * fniters + sets) * 2.0 * nrow * d
    wr = (3.0 * fniters + sets) * d
    rd += (3.0 * fniters + sets) * 2.0 * nrow * d
    wr += (3.0 * fniters + sets) * nrow * d
    rd += (fniters + sets) * (nnz * (d + i) + nrow * d)
    wr += (fniters + sets) * nrow * d
    for l in range(nlevels - 1):
        n_l, z_l = lv[l]
        rd += fniters * (2.0 * z_l * (d + i) + n_l * d)  # pre-smoother
        wr += fniters * n_l * d
        rd += fniters * (z_l * (d + i) + n_l * d)        # fine residual
        wr += fniters * z_l * d
        rd += fniters * (2.0 * z_l * (d + i) + n_l * d)  # post-smoother
        wr += fniters * z_l * d
    n_l, z_l = lv[-1]
    rd += fniters * (2.0 * z_l * (d + i) + n_l * d)
    wr += fniters * n_l * d
    return rd + wr


def compulsory_bytes(nx, ny, nz, nlevels=4, vb=8):
    """HBM bytes of one CG iteration when every matrix row is streamed once per use:

        sum_{l < L-1} [4.125 M_l + 13.625 N_l vb] + 2 M_{L-1} + 6 N_{L-1} vb + 12 nnz_0 + 136 N_0

    with M_l = nnz_l (vb + 4) (values + int32 columns). Per MG level: four
    Gauss-Seidel sweeps over the matrix plus the residual at the 1/8 injected
    rows (4.125 M_l) and the vector traffic of the sweeps, restriction and
    prolongation (13.625 N_l vb); the coarsest level does one symmetric sweep;
    the top level adds the CG SpMV (12 nnz_0) and 17 FP64 vector passes of the CG
    updates and dots (136 N_0). vb = 4 gives the FP32 V-cycle."""
    lv = level_sizes(nx, ny, nz, nlevels)
    b = 0.0
    for l in range(nlevels - 1):
        n_l, z_l = lv[l]
        b += 4.125 * z_l * (vb + 4) + 13.625 * n_l * vb
    n_l, z_l = lv[-1]
    b += 2.0 * z_l * (vb + 4) + 6.0 * n_l * vb
    n0, z0 = lv[0]
    b += 12.0 * z0 + 136.0 * n0
    return b


def index_bytes_per_row(pack=0):
    """Column-index bytes per row: 27 int32 columns (pack 0), or the packed
    index, one record per 128-row tile of 27 int32 bases and the form word
    followed by 27 x 128 offsets of `pack` bytes, 27.875 B (pack 1) or 54.875 B
    (2) a row, or by 27 x 128 sink bits (the diagonal form, pack 3), 4.25 B."""
    if pack == 3:
        return (28 * 4 + SLOTS * 4 * 4) / 128.0
    if pack:
        return (28 * 4 + SLOTS * 128 * pack) / 128.0
    return SLOTS * 4


def gs_phase_bytes(rows_in_phase, rows_in_level, vb=8, pack=0):
    """Algorithmic bytes of Gauss-Seidel colour phases that together updated
    `rows_in_phase` rows of a level with `rows_in_level` rows, per phase:
    27 ELL slots (value + column index: int32, or the packed index) and the
    right-hand side read, x written, for every row of the colour; and x of the
    seven other colours read once (each row of a colour neighbours all of them).
    For rows_in_phase = R summed over launches of one colour each, the
    other-colour reads are 7 R vb (the colours hold an eighth of the rows each)."""
    per_row = SLOTS * vb + index_bytes_per_row(pack) + 2 * vb
    return rows_in_phase * per_row + 7.0 * rows_in_phase * vb


def wave_sweep_bytes(rows_updated, rows_in_level, vb=8, pack=0):
    """Algorithmic bytes of Gauss-Seidel sweeps run as wavefront launches that
    together updated `rows_updated` rows, each launch a whole sweep of a level
    of `rows_in_level` rows (`rows_updated` / `rows_in_level` launches, rounded
    up: a backward sweep updates 7/8 of the rows): per updated row the 27 slots,
    the right-hand side read and x written; x read from DRAM once per sweep
    (the other colours' x stays in L2 between the phases of the wavefront)."""
    sweeps = -(-int(rows_updated) // int(rows_in_level)) if rows_in_level else 0
    return rows_updated * (SLOTS * vb + index_bytes_per_row(pack) + 2 * vb) + sweeps * rows_in_level * vb


def spmv_bytes(rows, vb=8, pack=0):
    """Algorithmic bytes of y = A x over `rows` rows: 27 values and column
    indices, x read once, y written."""
    return rows * (SLOTS * vb + index_bytes_per_row(pack) + 2 * vb)


def first_sweep_bytes(rows, vb=8):
    """Algorithmic bytes of the first forward sweeps (x = 0) that together
    updated `rows` rows, summed over whole sweeps (all eight colours): a phase
    reads only the slots of colours swept before it, 13 of the 27 per row on
    average (each neighbouring pair of colours once: 8 colours x 26 neighbours
    / 2 / 8), plus the diagonal value, the right-hand side, the x write and the
    swept colours' x (28 colour-eighths over 8 phases = 3.5 entries per row)."""
    return rows * (13 * (vb + 4) + vb + 2 * vb + 3.5 * vb)



def iteration_bytes(nx, ny, nz, vb=8, pack=(1, 1, 1, 1), nlevels=4, parts=False, rtz_fused=None,
                    wave=(0, 0, 0, 0)):
    """Algorithmic HBM bytes of one CG iteration as this library runs it, kernel
    by kernel (the floor its kernels move when each streams its data once):

    per level l with N_l rows, full-phase row bytes F_l = 36 vb + I_l (27
    values, the column index I_l = index_bytes_per_row(pack[l]), right-hand
    side, x written, the other seven colours' x), vb the V-cycle's value bytes
    (8 in the FP64 form, 4 in the FP32 V-cycle):

    * pre-smoother: the first forward sweep from x = 0 (first_sweep_bytes,
      13 slots with int32 columns on average) and the backward sweep's 7
      phases, 7/8 N_l F_l (the colour at the turn is not recomputed);
    * residual + restriction (levels above the coarsest): N_l/8 coarse rows of
      27 vb + I_l + 2 vb + 4 (rf read, rc written, the coarse row's index) and
      the fine x read once, N_l vb;
    * prolongation: N_l/8 (8 + 3 vb) (pair indices, xc read, xf read and written);
    * post-smoother: 15 phases, 15/8 N_l F_l;
    * coarsest level: one symmetric sweep (first sweep + 7 phases);
    * top level, always FP64: the CG SpMV fused with p'Ap (spmv_bytes with
      level 0's index) and the vector kernels: 64 B/row in the FP64 form
      (p and x update 40, r update 24) plus 16 B/row for an r'z pass of its
      own where the post-smoother does not accumulate r'z (level 0 on 8-bit
      or 16-bit offset records; rtz_fused=None derives that from pack[0]),
      and 96 B/row around the FP32 V-cycle (z widened with both flexible dots
      28, p and x update 40, r update with r narrowed 28).

    Levels with wave[l] set run the sweeps that start from nonzero x (the
    pre-smoother's backward sweep, both post-smoother sweeps) as wavefront
    launches: per sweep the updated rows' 29 vb + I_l and x read once, N_l vb,
    instead of 36 vb + I_l per updated row.

    With parts=True also returns the per-term split (GB)."""
    lv = level_sizes(nx, ny, nz, nlevels)
    split = {}
    total = 0.0
    for l, (n_l, _) in enumerate(lv):
        ib = index_bytes_per_row(pack[l])
        full = 36.0 * vb + ib
        wl = l < len(wave) and wave[l]
        # a sweep that starts from nonzero x and updates the fraction f of the rows
        sweep = (lambda f: f * n_l * (29.0 * vb + ib) + n_l * vb) if wl else (lambda f: f * n_l * full)
        b = first_sweep_bytes(n_l, vb) + sweep(7.0 / 8.0)
        if l < nlevels - 1:
            b += n_l / 8.0 * (27.0 * vb + ib + 2.0 * vb + 4.0) + n_l * vb
            b += n_l / 8.0 * (8.0 + 3.0 * vb)
            b += sweep(1.0) + sweep(7.0 / 8.0)
        split[f"level{l}"] = b / 1e9
        total += b
    n0 = lv[0][0]
    sp = spmv_bytes(n0, 8, pack[0])
    if rtz_fused is None:
        rtz_fused = pack[0] not in (1, 2)
    vec = (96.0 if vb != 8 else 64.0 if rtz_fused else 80.0) * n0
    split["spmv"] = sp / 1e9
    split["vectors"] = vec / 1e9
    total += sp + vec
    return (total, split) if parts else total
