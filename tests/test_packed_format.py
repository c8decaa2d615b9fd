"""The packed column format of the bulk-copy kernels, restated with numpy on the
host: the level's 27-slot ELL columns in colour order, one record per 128-row
tile (27 bases, 16-bit offsets, 0xFFFF for the zero sink). The device builds
the records in problem.cu (k_pack_cols) and decodes them in bulk.cuh
(stage_col); the GPU tests check that the decoded columns give the same bits as
the 32-bit ones. Here: the encoding round-trips, the stencil's colour order
keeps every tile's slot within a few hundred rows, and a matrix whose columns
scatter does not pack."""
import numpy as np
import pytest

ROWS = 128
SINK = 0xFFFF
MAX_SPAN = 0xFFFE


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


def pack(cols, n, pitch, sink):
    """(bases [tiles][27], offsets [tiles][27][128], packs, max span)."""
    t = pitch // ROWS
    c = np.where(np.arange(pitch) < n, cols, sink).reshape(27, t, ROWS).transpose(1, 0, 2)
    real = c != sink
    any_real = real.any(axis=2)
    lo = np.where(real, c, np.iinfo(np.int64).max).min(axis=2)
    hi = np.where(real, c, np.iinfo(np.int64).min).max(axis=2)
    span = np.where(any_real, hi - lo, 0)
    base = np.where(any_real, lo, 0)
    off = np.where(real, c - base[:, :, None], SINK)
    packs = bool((span <= MAX_SPAN).all())
    return base.astype(np.int32), off.astype(np.uint16), packs, int(span.max())


def unpack(base, off, sink):
    c = np.where(off == SINK, sink, base[:, :, None].astype(np.int64) + off)
    return c.transpose(1, 0, 2).reshape(27, -1)


@pytest.mark.parametrize("dims", [(16, 16, 16), (32, 32, 32), (16, 24, 40), (64, 64, 64)])
def test_stencil_columns_pack_and_round_trip(binding, dims):
    cols, n, pitch = colour_ell(binding, *dims)
    base, off, packs, span = pack(cols, n, pitch, n)
    assert packs
    # a tile is consecutive rows of one colour, and slot k of each is the
    # matching row of one neighbouring colour: the slot spans the tile's own
    # 128 rows (the sink aside), whatever the grid
    assert span == ROWS - 1
    back = unpack(base, off, n)
    assert np.array_equal(back[:, :n], cols[:, :n])
    # one record per tile: 27 bases + a padding word, 27 x 128 offsets
    assert base.shape[0] * (28 * 4 + 27 * ROWS * 2) == pitch // ROWS * 7024


def test_scattered_columns_do_not_pack(binding):
    cols, n, pitch = colour_ell(binding, 48, 48, 48)
    # a row whose columns jump across the whole level (as a rank's external
    # columns after its n interior rows do): that tile's slot spans > 65534
    far = cols.copy()
    far[14, 5] = n - 1
    far[14, 6] = 0
    assert n - 1 > MAX_SPAN
    _, _, packs, span = pack(far, n, pitch, n)
    assert not packs and span == n - 1
