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
