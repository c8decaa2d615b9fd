"""The packed column format of the bulk-copy kernels, restated with numpy on the
host: the level's 27-slot ELL columns in colour order, one record per 128-row
tile (27 bases and a word holding the record's form w, then either 27 x 128
offsets of w = 1 or 2 bytes, the all-ones offset marking the zero sink, or, for
the diagonal form w = 3, 27 x 128 sink bits with column = base + row
elsewhere). The diagonal form is taken where every tile's slots are diagonals,
else w = 1 where every tile's columns of each slot span at most 254, else 2
where they span at most 65534, else the level is not packed. The device builds
the records in problem.cu (k_pack_cols, k_pack_cols_diag) and decodes them in
bulk.cuh (stage_col); the GPU tests check that the decoded columns give the
same bits as the 32-bit ones and that each level gets the form predicted here
(packed_width). Here: the encodings round-trip, the stencil's colour order
makes every tile's slot a diagonal where colour blocks fill whole tiles, and a
matrix whose columns scatter does not pack."""
import numpy as np
import pytest

ROWS = 128


def sink_code(w):
    return 0xFF if w == 1 else 0xFFFF


def max_span(w):
    return 0xFE if w == 1 else 0xFFFE


def rec_bytes(w):
    return 28 * 4 + (27 * 4 * 4 if w == 3 else 27 * ROWS * w)


def colour_ell(binding, nx, ny, nz):
    """Columns [27][pitch] of the 27-point problem in the library's colour order
    (slot k = (sz+1)*9 + (sy+1)*3 + (sx+1), GenerateProblem_ref.cpp:152-172);
    a direction that leaves the grid holds the sink column n."""
    n = nx * ny * nz
    pitch = (n + 1 + 255) // 256 * 256
    n2o, _ = binding.colour_permutation(nx, ny, nz)
    o2n = np.empty(n, np.int64)
    o2n[n2o] = np.arange(n)
    ix, iy, iz = n2o % nx, (n2o // nx) % ny, n2o // (nx * ny)
    cols = np.full((27, pitch), n, np.int64)
    for sz in (-1, 0, 1):
        for sy in (-1, 0, 1):
            for sx in (-1, 0, 1):
                k = (sz + 1) * 9 + (sy + 1) * 3 + (sx + 1)
                jx, jy, jz = ix + sx, iy + sy, iz + sz
                ok = (jx >= 0) & (jx < nx) & (jy >= 0) & (jy < ny) & (jz >= 0) & (jz < nz)
                j = (jz * ny + jy) * nx + jx
                cols[k, :n][ok] = o2n[j[ok]]
    return cols, n, pitch


def pack(cols, n, pitch, sink, w=2):
    """(bases [tiles][27], offsets [tiles][27][128], packs, max span)."""
    t = pitch // ROWS
    c = np.where(np.arange(pitch) < n, cols, sink).reshape(27, t, ROWS).transpose(1, 0, 2)
    real = c != sink
    any_real = real.any(axis=2)
    lo = np.where(real, c, np.iinfo(np.int64).max).min(axis=2)
    hi = np.where(real, c, np.iinfo(np.int64).min).max(axis=2)
    span = np.where(any_real, hi - lo, 0)
    base = np.where(any_real, lo, 0)
    packs = bool((span <= max_span(w)).all())
    off = np.where(real, c - base[:, :, None], sink_code(w))
    if packs:
        off = off.astype(np.uint8 if w == 1 else np.uint16)
    return base.astype(np.int32), off, packs, int(span.max())


def unpack(base, off, sink, w=2):
    c = np.where(off == sink_code(w), sink, base[:, :, None].astype(np.int64) + off)
    return c.transpose(1, 0, 2).reshape(27, -1)


def pack_diag(cols, n, pitch, sink):
    """The diagonal form: (bases [tiles][27], sink bits [tiles][27][4] uint32,
    packs). A slot's base is column - row of its non-sink rows, which must agree."""
    t = pitch // ROWS
    c = np.where(np.arange(pitch) < n, cols, sink).reshape(27, t, ROWS).transpose(1, 0, 2)
    real = c != sink
    d = c - np.arange(ROWS)[None, None, :]
    lo = np.where(real, d, np.iinfo(np.int64).max).min(axis=2)
    hi = np.where(real, d, np.iinfo(np.int64).min).max(axis=2)
    any_real = real.any(axis=2)
    packs = bool(np.all(~any_real | (lo == hi)))
    base = np.where(any_real, lo, 0)
    sinks = (~real).reshape(t, 27, 4, 32)
    bits = (sinks.astype(np.uint64) << np.arange(32, dtype=np.uint64)).sum(axis=3).astype(np.uint32)
    return base.astype(np.int64), bits, packs


def unpack_diag(base, bits, sink):
    t = base.shape[0]
    sinks = ((bits[:, :, :, None] >> np.arange(32, dtype=np.uint32)) & 1).reshape(t, 27, ROWS).astype(bool)
    c = np.where(sinks, sink, base[:, :, None] + np.arange(ROWS)[None, None, :])
    return c.transpose(1, 0, 2).reshape(27, -1)


def packed_width(binding, nx, ny, nz, diagonal=True):
    """The column form the library gives a single-rank level of this grid: 3
    (diagonal), 1, 2 (offset bytes), or 0 (not packed); diagonal=False: as with
    HPCG_B200_PACKED=8."""
    cols, n, pitch = colour_ell(binding, nx, ny, nz)
    if diagonal and pack_diag(cols, n, pitch, n)[2]:
        return 3
    for w in (1, 2):
        if pack(cols, n, pitch, n, w)[2]:
            return w
    return 0


@pytest.mark.parametrize("w", [1, 2])
@pytest.mark.parametrize("dims", [(16, 16, 16), (32, 32, 32), (16, 24, 40), (64, 64, 64)])
def test_stencil_columns_pack_and_round_trip(binding, dims, w):
    cols, n, pitch = colour_ell(binding, *dims)
    base, off, packs, span = pack(cols, n, pitch, n, w)
    assert packs
    # a tile is consecutive rows of one colour, and slot k of each is the
    # matching row of one neighbouring colour: the slot spans the tile's own
    # 128 rows (the sink aside), whatever the grid, as long as every colour
    # block is a whole number of tiles
    assert span == ROWS - 1
    back = unpack(base, off, n, w)
    assert np.array_equal(back[:, :n], cols[:, :n])
    # one record per tile: 27 bases + the width word, 27 x 128 offsets
    assert base.shape[0] * rec_bytes(w) == pitch // ROWS * (3568 if w == 1 else 7024)


@pytest.mark.parametrize("dims", [(16, 16, 16), (32, 32, 32), (16, 24, 40), (64, 64, 64)])
def test_stencil_columns_are_tile_diagonals(binding, dims):
    """Where every colour block is a whole number of tiles, each slot's columns
    across a tile are one diagonal (column = base + row) apart from the sink:
    the diagonal form holds them in 4.25 bytes a row and decodes every column."""
    cols, n, pitch = colour_ell(binding, *dims)
    base, bits, packs = pack_diag(cols, n, pitch, n)
    assert packs
    back = unpack_diag(base, bits, n)
    assert np.array_equal(back[:, :n], cols[:, :n])
    assert np.all(back[:, n:] == n)
    assert base.shape[0] * rec_bytes(3) == pitch // ROWS * 544


@pytest.mark.parametrize("dims,form,width", [((24, 24, 24), 2, 2), ((48, 48, 48), 3, 1), ((8, 8, 8), 2, 2),
                                             ((4, 4, 4), 1, 1), ((12, 12, 12), 2, 2), ((64, 32, 16), 3, 1)])
def test_form_follows_the_colour_blocks(binding, dims, form, width):
    """The diagonal form holds every level whose colour blocks fill whole
    128-row tiles; 8-bit offsets (the form without it) hold those and every
    level of at most 255 columns; a tile that straddles two colour blocks spans
    the distance between their neighbour colours, which at 24^3 or 8^3 needs
    16 bits."""
    assert packed_width(binding, *dims) == form
    assert packed_width(binding, *dims, diagonal=False) == width


def test_scattered_columns_do_not_pack(binding):
    cols, n, pitch = colour_ell(binding, 48, 48, 48)
    # a row whose columns jump across the whole level (as a rank's external
    # columns after its n interior rows do): that tile's slot spans > 65534
    far = cols.copy()
    far[14, 5] = n - 1
    far[14, 6] = 0
    assert n - 1 > max_span(2)
    for w in (1, 2):
        _, _, packs, span = pack(far, n, pitch, n, w)
        assert not packs and span == n - 1
    assert not pack_diag(far, n, pitch, n)[2]
    # a jump of 300 rows: off the diagonal, too far for 8 bits, near enough for 16
    near = cols.copy()
    near[14, 5] = cols[14, 5] + 300
    assert not pack_diag(near, n, pitch, n)[2]
    assert pack(near, n, pitch, n, 1)[2] is False
    assert pack(near, n, pitch, n, 2)[2] is True
