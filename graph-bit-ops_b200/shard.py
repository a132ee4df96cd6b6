"""Block-row sharding of BFS across GPUs, one process per GPU.

Each rank holds the block rows [R0, R1) of the graph (all columns) as its own
B2SR graph.  A level is one pull step per shard against the whole frontier,
a sum of the new-vertex counts (the loop ends at zero) and an all-gather of
the shards' next-frontier words (n/8 bytes in all).  The loop and the data
plane are the library's (gbo_bfs_sharded over an NCCL communicator made by
gbo_nccl_comm_create); this module only partitions the rows and holds the
handles.  The NCCL unique id (128 bytes, from gbo_nccl_unique_id on one rank)
reaches the other ranks over any host channel the caller has.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

import gbo


def partition_rows(rowptr, nrows: int, nshards: int, tile_bits: int) -> list[int]:
    """Row boundaries 0 = b_0 <= ... <= b_S = nrows, multiples of the tile
    width except the last, splitting the stored entries about evenly."""
    b = tile_bits
    nbr = (nrows + b - 1) // b
    rowptr = np.asarray(rowptr, np.int64)
    ends = np.minimum(np.arange(1, nbr + 1) * b, nrows)
    cum = rowptr[ends]  # entries up to the end of each block row
    total = int(rowptr[nrows])
    cuts = [0]
    for s in range(1, nshards):
        R = int(np.searchsorted(cum, total * s / nshards, side="left")) + 1
        cuts.append(max(cuts[-1], min(R, nbr)))
    cuts.append(nbr)
    return [min(R * b, nrows) for R in cuts]


def shard_csr(csr: gbo.Csr, r0: int, r1: int) -> gbo.Csr:
    """The rows [r0, r1) of a CSR, every column."""
    a, e = int(csr.rowptr[r0]), int(csr.rowptr[r1])
    return gbo.Csr(csr.rowptr[r0:r1 + 1] - a, csr.colind[a:e], r1 - r0, csr.ncols)


def nccl_unique_id() -> bytes:
    """A new NCCL unique id (call on one rank, hand the bytes to all)."""
    buf = C.create_string_buffer(128)
    gbo.check(gbo.lib().gbo_nccl_unique_id(buf), "nccl_unique_id")
    return buf.raw


class NcclComm:
    """The library's NCCL data plane for one rank (its device current)."""

    def __init__(self, world: int, rank: int, uid: bytes):
        self.h = C.c_void_p()
        gbo.check(gbo.lib().gbo_nccl_comm_create(world, rank, uid, C.byref(self.h)), "nccl_comm_create")

    def close(self):
        if self.h:
            gbo.lib().gbo_nccl_comm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BfsShard:
    """One rank's block rows of the graph and the sharded BFS over them."""

    def __init__(self, csr: gbo.Csr, bounds: list[int], rank: int, tile_bits: int = 32):
        self.b, self.n = tile_bits, csr.nrows
        self.bounds = [int(x) for x in bounds]
        self.rank, self.world = rank, len(bounds) - 1
        self.r0, self.r1 = self.bounds[rank], self.bounds[rank + 1]
        self.g = gbo.Graph.from_csr(shard_csr(csr, self.r0, self.r1), tile_bits)
        self.level = gbo.DeviceBuffer(4 * max(self.r1 - self.r0, 1))

    def bfs(self, src: int, comm, stream=None) -> int:
        """BFS from `src` over all ranks (every rank calls it); returns the
        number of levels.  `comm` is an NcclComm or a gbo_shard_comm pointer."""
        h = comm.h if isinstance(comm, NcclComm) else comm
        bounds = (C.c_int * (self.world + 1))(*self.bounds)
        depth = C.c_int(0)
        gbo.check(gbo.lib().gbo_bfs_sharded(self.g.h, self.rank, self.world, bounds, int(src), self.level.ptr,
                                            C.byref(depth), h, stream), "bfs_sharded")
        return depth.value

    def levels(self) -> np.ndarray:
        """int32 levels of this rank's rows after bfs()."""
        return self.level.to_numpy(np.int32, self.r1 - self.r0)

    def free(self) -> None:
        if self.g is not None:
            self.g.free()
            self.g = None
