"""Block-row sharded BFS (gbo_bfs_shard_level driven by shard.py): the shards'
levels, put side by side, are the whole graph's BFS levels.  The shards run
in one process on one GPU (the exchange is a device copy); the multi-process
path is covered on the CPU in tests/test_dist.py."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def shard_mod(gbo):
    sys.path.insert(0, os.path.dirname(gbo.__file__))
    import shard

    return shard


@pytest.mark.parametrize("b", [8, 32, 64])
@pytest.mark.parametrize("nshards", [1, 3])
def test_sharded_bfs_matches_bfs(gbo, orc, gpu, shard_mod, b, nshards):
    import torch

    csr = gbo.gen_rmat(12, 16, seed=9)
    bounds = shard_mod.partition_rows(csr.rowptr, csr.nrows, nshards, b)
    shards = [shard_mod.BfsShard(csr, bounds, s, b) for s in range(nshards)]
    g = gbo.Graph.from_csr(csr, b)
    for src in (0, 777, csr.nrows - 1):
        shard_mod.run_local(shards, src)
        got = torch.cat([sh.levels() for sh in shards]).cpu().numpy()
        want, _ = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, src)
        assert np.array_equal(got, want), (b, nshards, src)
        assert np.array_equal(g.bfs(src)[0], want)
    for sh in shards:
        sh.free()
    g.free()
