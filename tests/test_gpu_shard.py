"""Block-row sharded BFS on the GPU (gbo_bfs_sharded): the shards' levels,
put side by side, are the whole graph's BFS levels.  With one GPU the ranks
are host threads of one process whose data plane copies device buffers
between them (only host-side waits: no kernel waits on another rank), and
one rank runs over the library's NCCL communicator.  The multi-process loop
is covered on the CPU in tests/test_dist.py."""
import ctypes as C
import os
import sys
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def shard_mod(gbo):
    sys.path.insert(0, os.path.dirname(gbo.__file__))
    import shard

    return shard


class ThreadComm:
    """Data plane between `world` threads of this process: a summed count and
    an all-gather that copies every rank's device bytes into every rank's
    receive buffer."""

    def __init__(self, gbo, world):
        self.gbo, self.world = gbo, world
        self.bar = threading.Barrier(world, timeout=120)
        self.vals = [0] * world
        self.sends = [0] * world
        self.structs = []
        for r in range(world):
            ar = gbo.SHARD_ALLREDUCE_FN(lambda u, v, r=r: self._allreduce(r, v))
            ag = gbo.SHARD_ALLGATHER_FN(lambda u, s, d, n, st, r=r: self._allgather(r, s, d, n, st))
            self.structs.append(gbo.ShardComm(None, ar, ag))

    def _allreduce(self, r, value):
        self.vals[r] = value[0]
        self.bar.wait()
        value[0] = sum(self.vals)
        self.bar.wait()
        return 0

    def _allgather(self, r, d_send, d_recv, nbytes, stream):
        self.sends[r] = d_send
        self.gbo.lib().gbo_stream_sync(stream)  # this rank's part is written
        self.bar.wait()
        for s, src in enumerate(self.sends):
            st = self.gbo.lib().gbo_memcpy_d2d(d_recv + s * nbytes, src, nbytes, stream)
            if st:
                return st
        self.gbo.lib().gbo_stream_sync(stream)  # nobody reuses a send buffer early
        self.bar.wait()
        return 0

    def ptr(self, r):
        return C.addressof(self.structs[r])


@pytest.mark.parametrize("b", [8, 32, 64])
@pytest.mark.parametrize("nshards", [1, 3])
def test_sharded_bfs_matches_bfs(gbo, orc, gpu, shard_mod, b, nshards):
    csr = gbo.gen_rmat(12, 16, seed=9)
    bounds = shard_mod.partition_rows(csr.rowptr, csr.nrows, nshards, b)
    shards = [shard_mod.BfsShard(csr, bounds, s, b) for s in range(nshards)]
    comm = ThreadComm(gbo, nshards)
    streams = [gbo.Stream() for _ in range(nshards)]
    for src in (0, 777, csr.nrows - 1):
        depths = [None] * nshards
        errs = []

        def run(r):
            try:
                depths[r] = shards[r].bfs(src, comm.ptr(r), streams[r].ptr)
            except Exception as e:  # reported below
                errs.append(e)

        ths = [threading.Thread(target=run, args=(r,)) for r in range(nshards)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        assert not errs, errs
        got = np.concatenate([sh.levels() for sh in shards])
        want, d = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, src)
        assert np.array_equal(got, want), (b, nshards, src)
        assert depths == [d] * nshards
    for sh in shards:
        sh.free()


def test_sharded_bfs_over_nccl_one_rank(gbo, orc, gpu, shard_mod):
    """The library's NCCL data plane with a single rank (the only GPU)."""
    csr = gbo.gen_rmat(11, 16, seed=3)
    bounds = [0, csr.nrows]
    sh = shard_mod.BfsShard(csr, bounds, 0, 32)
    comm = shard_mod.NcclComm(1, 0, shard_mod.nccl_unique_id())
    for src in (1, 1000):
        depth = sh.bfs(src, comm)
        want, d = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, src)
        assert np.array_equal(sh.levels(), want) and depth == d
    comm.close()
    sh.free()


def test_sharded_bfs_argument_checks(gbo, gpu, shard_mod):
    csr = gbo.gen_rmat(9, 8, seed=1)
    sh = shard_mod.BfsShard(csr, [0, csr.nrows], 0, 32)
    comm = ThreadComm(gbo, 1)
    bad = (C.c_int * 2)(0, csr.nrows + 5)  # does not match the shard's rows
    depth = C.c_int(0)
    st = gbo.lib().gbo_bfs_sharded(sh.g.h, 0, 1, bad, 0, sh.level.ptr, C.byref(depth), comm.ptr(0), None)
    assert st == gbo.GBO_ERR_INVALID
    good = (C.c_int * 2)(0, csr.nrows)
    st = gbo.lib().gbo_bfs_sharded(sh.g.h, 0, 1, good, csr.nrows, sh.level.ptr, C.byref(depth), comm.ptr(0), None)
    assert st == gbo.GBO_ERR_INVALID  # source out of range
    sh.free()
