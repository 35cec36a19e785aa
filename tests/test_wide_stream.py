"""Index arithmetic of the wide-tile likelihood's window stream (no GPU).

The wide tiles (csrc/fbp_lik_tcw.cuh) lay a pass's listed windows end to end:
listed window i starts at stream position i*L + R_i*(L-1), with R_i the number
of runs of consecutive windows before it (k_ws_pos).  A tile is 2048
positions; the kernel stages 2048 + 16*ceil((L+7)/16) positions (the lags of
its last outputs) and builds a table of the listed windows that meet them.
Its error paths assume two facts about that table:
  * the first listed window at or before every tile start is known
    (first[q]; error 16 otherwise), and
  * at most kWTwMax = 136 listed windows meet a tile's staged positions for
    any L >= 16 (error 15 otherwise).
These tests restate the stream's formulas and check both facts, and that
every kept output lies in exactly one tile, on random window lists."""
import numpy as np
import pytest

K_WPOS = 2048
K_WTWMAX = 136


def nkc(L):
    return (L + 7 + 15) // 16


def stream(win, L):
    """pos, first, n_stiles as k_ws_breaks / compaction / k_ws_pos compute them."""
    m = len(win)
    brk = np.ones(m, bool)
    brk[1:] = win[1:] != win[:-1] + 1
    runs_before = np.cumsum(brk) - 1                  # R_i
    pos = np.arange(m, dtype=np.int64) * L + runs_before * (L - 1)
    n_stiles = (int(pos[-1]) + L + K_WPOS - 1) // K_WPOS if m else 0
    first = {}
    for i in range(m):
        nxt = pos[i] + L + ((L - 1) if (i + 1 < m and brk[i + 1]) else 0) if i + 1 < m else None
        qt = (int(pos[i]) + K_WPOS - 1) // K_WPOS     # the one tile start in [pos_i, next)
        if nxt is not None:
            if qt * K_WPOS < nxt:
                first[qt] = i
        elif qt * K_WPOS < pos[i] + L:
            first[qt] = i
    return pos, first, n_stiles


def window_lists(rng, W, density):
    """Sorted distinct window ids: runs and isolated windows."""
    keep = rng.random(W) < density
    if not keep.any():
        keep[rng.integers(W)] = True
    return np.nonzero(keep)[0].astype(np.int64)


@pytest.mark.parametrize("L", [16, 31, 41, 61, 101, 150, 190])
@pytest.mark.parametrize("density", [1.0, 0.9, 0.5, 0.1, 0.01])
def test_every_tile_has_a_first_entry_and_a_bounded_table(L, density):
    rng = np.random.Generator(np.random.PCG64(1000 * L + int(100 * density)))
    px = K_WPOS + 16 * nkc(L)
    for _ in range(4):
        W = int(rng.integers(50, 3000))
        win = window_lists(rng, W, density)
        pos, first, n_stiles = stream(win, L)
        assert np.all(np.diff(pos) >= L)              # windows never share positions
        for q in range(n_stiles):
            Q0 = q * K_WPOS
            assert q in first, (L, density, q)
            i_lo = first[q]
            assert pos[i_lo] <= Q0                    # tpos[0] <= 0 in the kernel's table
            touching = np.count_nonzero((np.arange(len(win)) >= i_lo) & (pos < Q0 + px))
            assert touching <= K_WTWMAX, (L, density, touching)


@pytest.mark.parametrize("L", [16, 61, 101])
def test_every_kept_output_lies_in_one_tile(L):
    rng = np.random.Generator(np.random.PCG64(77 + L))
    win = window_lists(rng, 1500, 0.3)
    pos, first, n_stiles = stream(win, L)
    covered = np.zeros(n_stiles * K_WPOS, np.int32)
    for p in pos:
        covered[p:p + L] += 1                         # the L kept outputs of a listed window
    assert covered.max() == 1
    assert covered.sum() == len(win) * L
