"""Tile-width tuner: the model ranks widths by the bytes of one sweep over
the packing (checked against the packed graphs' tile counts), the timed mode
returns the width with the smallest measured time."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
WIDTHS = (4, 8, 16, 32, 64)


def _sweep_bytes(nblk, b, nrows):
    wb = max(1, b // 8)
    return nblk * (b * wb + 4) + 4 * ((nrows + b - 1) // b + 1)


@pytest.mark.parametrize("name", ["rmat12", "mesh64", "er2000"])
def test_model_matches_packed_tile_counts(gbo, gpu, name):
    csr = {"rmat12": lambda: gbo.gen_rmat(12, 16, seed=0), "mesh64": lambda: gbo.gen_king_mesh(64),
           "er2000": lambda: gbo.gen_er(2000, 0.004, 1)}[name]()
    for op, flags in ((gbo.TUNE_BMV, 0), (gbo.TUNE_TC, gbo.FLAG_LOWER)):
        best, cost = gbo.tune_tile_width(csr, op, gbo.TUNE_MODEL)
        for b in WIDTHS:
            nblk = int(gbo.Graph.from_csr(csr, b, flags).info().nblocks)
            assert cost[b] == _sweep_bytes(nblk, b, csr.nrows), (name, op, b)
        allowed = WIDTHS if op == gbo.TUNE_BMV else WIDTHS[1:]
        assert best == min(allowed, key=lambda b: cost[b])


def test_timed_picks_fastest(gbo, gpu):
    csr = gbo.gen_rmat(13, 16, seed=3)
    for op in (gbo.TUNE_BMV, gbo.TUNE_BFS, gbo.TUNE_TC):
        best, ms = gbo.tune_tile_width(csr, op, gbo.TUNE_TIMED)
        allowed = WIDTHS if op != gbo.TUNE_TC else WIDTHS[1:]
        assert all(ms[b] > 0 and math.isfinite(ms[b]) for b in allowed)
        assert best == min(allowed, key=lambda b: ms[b])


def test_bfs_model_counts_row_word_slices_at_32(gbo, gpu):
    """For BFS at b = 32 the model prices the row-word slices: 8 bytes per
    distinct (row, column / 32) pair and 8 per row; other widths stay tiles."""
    csr = gbo.gen_rmat(12, 16, seed=5)
    best, cost = gbo.tune_tile_width(csr, gbo.TUNE_BFS, gbo.TUNE_MODEL)
    rows = np.repeat(np.arange(csr.nrows), np.diff(csr.rowptr))
    words = len(set(zip(rows.tolist(), (csr.colind // 32).tolist())))
    assert cost[32] == 8 * words + 8 * (csr.nrows + 1)
    for b in (4, 8, 16, 64):
        nblk = int(gbo.Graph.from_csr(csr, b).info().nblocks)
        assert cost[b] == _sweep_bytes(nblk, b, csr.nrows), b
    assert best == min(WIDTHS, key=lambda b: cost[b])
