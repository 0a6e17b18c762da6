"""Host-side checks of the batched kernel's band layout and window indexing
(jellyfih_b200/csrc/jf_batched.cu), restated here in Python:

* the band cut of sort_scan_kernel (quantile rows of the per-row cost,
  clamped to band_cap rows per band and to what the later bands can still
  cover) always yields monotone bands that cover the grid, none longer than
  band_cap, for any row costs;
* every shared-memory index chunk_kernel forms from such a layout stays in
  its window: the register-block flush rows, the halo push / pull rows and
  their owners' rows, the remote rows of generic scatters and gathers, and
  the grid-update rows;
* the TMEM node blocks of chunk_kernel<true> (544 .. 768 threads): every
  warp's 48 columns lie inside the CTA's allocation, warps of one lane
  quadrant never share a column, and every tcgen05.ld / tcgen05.st starts at
  a multiple of its width in columns.
"""
import numpy as np
import pytest

K_HALO_LO, K_HALO_HI = 1, 3  # window rows below / above a band
K_ROW_COST = 40


def band_cap_for(ny, cs, nx=128, planes=5, slack_bytes=128 * 1024):
    """jf_create's band_cap: ceil(ny / CS) rows plus a quarter while the window fits."""
    band_h = (ny + cs - 1) // cs
    fit = slack_bytes // (4 * planes * nx) - (K_HALO_LO + K_HALO_HI)
    bc = min(band_h + band_h // 4, fit)
    bc = max(bc, band_h)
    return min(bc, ny)


def cut_bands(row_cost, cs, band_cap):
    """sort_scan_kernel's band starts (brow[0 .. CS])."""
    ny = len(row_cost)
    total = int(np.sum(row_cost))
    brow = [0]
    pre, y = 0, 0
    for r in range(1, cs):
        target = total * r // cs
        while y < ny and pre + row_cost[y] // 2 < target:
            pre += row_cost[y]
            y += 1
        b = y
        b = min(b, brow[r - 1] + band_cap)
        b = max(b, ny - (cs - r) * band_cap)
        b = max(b, brow[r - 1])
        b = min(b, ny)
        while y > b:
            y -= 1
            pre -= row_cost[y]
        while y < b:
            pre += row_cost[y]
            y += 1
        brow.append(b)
    brow.append(ny)
    return brow


def owner_of(brow, j):
    cs = len(brow) - 1
    o = 0
    while o + 1 < cs and brow[o + 1] <= j:
        o += 1
    return o


def owner_row(brow, j, o):
    return j - (brow[o] - K_HALO_LO)


def check_layout(brow, ny, band_cap):
    cs = len(brow) - 1
    WR = band_cap + K_HALO_LO + K_HALO_HI
    assert brow[0] == 0 and brow[-1] == ny
    assert all(brow[r] <= brow[r + 1] for r in range(cs))
    assert all(brow[r + 1] - brow[r] <= band_cap for r in range(cs))
    for r in range(cs):
        row0, own_hi = brow[r], brow[r + 1]
        n_own = own_hi - row0
        win0 = row0 - K_HALO_LO
        VR = n_own + K_HALO_LO + K_HALO_HI
        assert VR <= WR

        def remote_ok(j):
            o = owner_of(brow, j)
            wr = owner_row(brow, j, o)
            assert brow[o] <= j < brow[o + 1], (brow, r, j)
            assert 1 <= wr <= brow[o + 1] - brow[o]

        # register-block flush: rows cy-1 .. cy+2 of the band's cells, in the window
        for cy in range(row0, own_hi):
            for J in range(4):
                assert 0 <= cy - 1 + J - win0 < VR
        # halo rows: pushed to / pulled from their owners' own rows
        for h in range(VR - n_own):
            wr = 0 if h == 0 else n_own + h
            j = win0 + wr
            if 0 <= j < ny:
                assert owner_of(brow, j) != r or n_own == 0
                remote_ok(j)
        # generic scatters / gathers: stencil rows anywhere in the grid
        for j in range(ny):
            if not (0 <= j - win0 < VR):
                remote_ok(j)
        # grid update: window rows 1 .. n_own
        for wr in range(K_HALO_LO, K_HALO_LO + n_own):
            assert win0 + wr < own_hi


@pytest.mark.parametrize("cs", [1, 2, 3, 4, 8, 16])
@pytest.mark.parametrize("ny", [16, 40, 128, 256])
def test_band_cut_and_window_indices(cs, ny):
    rng = np.random.default_rng(cs * 1000 + ny)
    cap = band_cap_for(ny, cs)
    for trial in range(60):
        kind = trial % 4
        if kind == 0:
            cost = rng.integers(0, 5000, ny)
        elif kind == 1:  # all work in a few rows
            cost = np.zeros(ny, np.int64)
            cost[rng.integers(0, ny, 3)] = rng.integers(1, 10 ** 6, 3)
        elif kind == 2:  # empty grid: only the grid-update cost
            cost = np.zeros(ny, np.int64)
        else:  # a dense bottom half, as a settled water column
            cost = np.where(np.arange(ny) < ny // 2, 4000, 0)
        cost = (np.asarray(cost, np.int64) + K_ROW_COST).tolist()
        brow = cut_bands(cost, cs, cap)
        check_layout(brow, ny, cap)


def test_fixed_bands_are_valid():
    """Grids taller than the dynamic limit keep equal bands of ceil(ny / CS) rows."""
    for ny, cs in [(2048, 16), (1100, 8)]:
        band_h = (ny + cs - 1) // cs
        brow = [min(r * band_h, ny) for r in range(cs)] + [ny]
        check_layout(brow, ny, band_h)


# tcgen05 accesses of one warp's block, relative to its first column
# (tm_zero48, tm_load_rows01 / tm_store_rows01, tm_load_rows23 / tm_store_rows23):
# (column offset, width in columns)
TMEM_ACCESSES = [(0, 16), (16, 16), (32, 16),  # zero
                 (0, 16), (16, 8),             # block rows 0 and 1
                 (24, 8), (32, 16)]            # block rows 2 and 3


def tmem_layout(n_warps):
    """chunk_kernel<true>'s allocation (a power of two >= 32 columns covering
    48 columns per warp of a lane quadrant) and warp w's (lane quadrant, first
    column)."""
    per_quad = (n_warps + 3) >> 2
    cols = 32
    while cols < 48 * per_quad:
        cols <<= 1
    return cols, [(w & 3, 48 * (w >> 2)) for w in range(n_warps)]


@pytest.mark.parametrize("threads", range(544, 769, 32))
def test_tmem_node_blocks_fit_and_are_aligned(threads):
    n_warps = threads // 32
    cols, warps = tmem_layout(n_warps)
    assert cols in (256, 512)  # tcgen05.alloc: a power of two, 32 .. 512 columns
    used = {}
    for w, (quad, base) in enumerate(warps):
        assert 0 <= quad < 4  # lanes 32 quad .. 32 quad + 31 of 128
        for off, width in TMEM_ACCESSES:
            start = base + off
            assert start % width == 0, (w, off, width)
            assert start + width <= cols, (w, off, width)
        for c in range(base, base + 48):
            assert (quad, c) not in used, (w, used.get((quad, c)))
            used[(quad, c)] = w
    # the accesses of one block cover exactly its 48 columns
    load_store = TMEM_ACCESSES[3:]
    assert sorted(c for off, width in load_store for c in range(off, off + width)) == list(range(48))
