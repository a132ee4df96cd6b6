"""Host side of the block-row sharded BFS: the row partition."""
import os
import sys

import numpy as np
import pytest


@pytest.fixture(scope="module")
def shard_mod(gbo):
    sys.path.insert(0, os.path.dirname(gbo.__file__))
    import shard

    return shard


def test_partition_rows_balances_entries(shard_mod, gbo):
    csr = gbo.gen_rmat(12, 16, seed=9)
    for b in (8, 32):
        bounds = shard_mod.partition_rows(csr.rowptr, csr.nrows, 4, b)
        assert bounds[0] == 0 and bounds[-1] == csr.nrows
        assert all(x % b == 0 for x in bounds[:-1]) and bounds == sorted(bounds)
        parts = np.diff(csr.rowptr[bounds])
        ends = np.minimum(np.arange(1, (csr.nrows + b - 1) // b + 1) * b, csr.nrows)
        widest = int(np.diff(np.concatenate([[0], csr.rowptr[ends]])).max())  # entries of one block row
        assert parts.max() <= csr.nnz / 4 + widest


@pytest.mark.parametrize("nshards", [1, 2, 7, 200])
def test_partition_rows_edge_cases(shard_mod, gbo, nshards):
    """More shards than block rows, a graph whose entries sit in one block
    row, an empty graph and a row count that is not a multiple of the tile:
    the bounds still cover [0, n) in order, on tile rows, and the shards'
    CSRs put every entry back."""
    b = 32
    n = 1000  # 31.25 block rows
    hub = gbo.csr_from_edges(np.zeros(n - 1, np.int32), np.arange(1, n, dtype=np.int32), n, False, True)
    empty = gbo.Csr(np.zeros(n + 1, np.int64), np.zeros(0, np.int32), n, n)
    for csr in (hub, empty, gbo.gen_er(n, 0.01, 3)):
        bounds = shard_mod.partition_rows(csr.rowptr, csr.nrows, nshards, b)
        assert len(bounds) == nshards + 1
        assert bounds[0] == 0 and bounds[-1] == n and bounds == sorted(bounds)
        assert all(x % b == 0 or x == n for x in bounds)
        parts = [shard_mod.shard_csr(csr, bounds[s], bounds[s + 1]) for s in range(nshards)]
        assert sum(p.nrows for p in parts) == n
        assert np.array_equal(np.concatenate([p.colind for p in parts]), csr.colind)
        for p in parts:
            assert p.rowptr[0] == 0 and p.rowptr[-1] == len(p.colind) and p.ncols == n
