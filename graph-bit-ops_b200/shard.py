"""Block-row sharding of BFS across GPUs, one process per GPU.

Each rank holds the block rows [R0, R1) of the graph (all columns) as its own
B2SR graph; a level is one pull step per shard against the whole frontier
(gbo_bfs_shard_level) followed by an all-gather of the shards' next-frontier
words (n/8 bytes in all) and an all-reduce of the new-vertex counts, which
ends the loop when it is zero.  Shards are balanced by stored entries with
boundaries on tile rows.  The data movement is torch.distributed (NCCL over
NVLink between GPUs); the step itself is the library's kernel.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

import gbo

_TORCH_WORD = {4: torch.uint8, 8: torch.uint8, 16: torch.int16, 32: torch.int32, 64: torch.int64}


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


class BfsShard:
    """One rank's block rows of the graph and its BFS state on `device`."""

    def __init__(self, csr: gbo.Csr, bounds: list[int], rank: int, tile_bits: int = 32,
                 device: str | torch.device = "cuda"):
        b = tile_bits
        self.b, self.n = b, csr.nrows
        self.r0, self.r1 = bounds[rank], bounds[rank + 1]
        self.R0 = self.r0 // b
        self.nbr = (self.r1 - self.r0 + b - 1) // b
        self.nbr_all = (self.n + b - 1) // b
        self.word_bounds = [r // b if r < self.n else self.nbr_all for r in bounds]
        self.device = torch.device(device)
        dt = _TORCH_WORD[b]
        self.front = torch.zeros(self.nbr_all, dtype=dt, device=self.device)
        self.visited = torch.zeros(max(self.nbr, 1), dtype=dt, device=self.device)
        self.next = torch.zeros(max(self.nbr, 1), dtype=dt, device=self.device)
        self.level = torch.full((max(self.r1 - self.r0, 1),), -1, dtype=torch.int32, device=self.device)
        self.g = self._build(shard_csr(csr, self.r0, self.r1)) if self.device.type == "cuda" else None

    def _build(self, part: gbo.Csr):
        return gbo.Graph.from_csr(part, self.b)

    def _bit(self, v: int) -> int:
        return 1 << (self.b - 1 - v % self.b)

    def reset(self, src: int) -> None:
        """Level 0: the source in every rank's frontier, in its owner's state."""
        self.front.zero_()
        self.visited.zero_()
        self.next.zero_()
        self.level.fill_(-1)
        w = self._signed(self._bit(src))
        self.front[src // self.b] = w
        if self.r0 <= src < self.r1:
            self.level[src - self.r0] = 0
            self.visited[src // self.b - self.R0] = w

    def _signed(self, bits: int) -> int:
        """A word's bit pattern as the value of the signed torch element type."""
        width = {4: 8, 8: 8, 16: 16, 32: 32, 64: 64}[self.b]
        if self.b <= 8:
            return bits
        return bits - (1 << width) if bits >> (width - 1) else bits

    def level_step(self, lvl: int) -> int:
        """One pull level over this shard: next-frontier words, visited,
        levels; the number of new vertices."""
        cnt = C.c_uint64(0)
        gbo.check(gbo.lib().gbo_bfs_shard_level(self.g.h, self.front.data_ptr(), self.visited.data_ptr(),
                                                 self.level.data_ptr(), lvl, self.next.data_ptr(),
                                                 C.byref(cnt), None), "bfs_shard_level")
        return int(cnt.value)

    def place(self, parts: list[torch.Tensor]) -> None:
        """The next frontier: every shard's next words at its block rows."""
        for s, part in enumerate(parts):
            lo, hi = self.word_bounds[s], self.word_bounds[s + 1]
            self.front[lo:hi] = part[: hi - lo]

    def levels(self) -> torch.Tensor:
        return self.level[: self.r1 - self.r0]

    def free(self) -> None:
        if self.g is not None:
            self.g.free()
            self.g = None


def run_distributed(shard: BfsShard, src: int, group=None) -> int:
    """BFS from `src` over all ranks of `group` (one shard each); returns
    the number of levels.  Every rank takes the same collective steps."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    width = max(b - a for a, b in zip(shard.word_bounds[:-1], shard.word_bounds[1:]))
    width = max(width, 1)
    shard.reset(src)
    lvl = 0
    while True:
        cnt = torch.tensor([shard.level_step(lvl)], dtype=torch.int64, device=shard.device)
        dist.all_reduce(cnt, group=group)
        if int(cnt.item()) == 0:
            return lvl + 1
        mine = torch.zeros(width, dtype=shard.next.dtype, device=shard.device)
        k = shard.word_bounds[dist.get_rank(group) + 1] - shard.word_bounds[dist.get_rank(group)]
        mine[:k] = shard.next[:k]
        gathered = torch.empty(world * width, dtype=shard.next.dtype, device=shard.device)
        dist.all_gather_into_tensor(gathered.view(torch.uint8), mine.view(torch.uint8), group=group)
        shard.place([gathered[s * width:(s + 1) * width] for s in range(world)])
        lvl += 1


def run_local(shards: list[BfsShard], src: int) -> int:
    """The same loop with every shard in this process (one device): the
    exchange is a copy on the device."""
    for sh in shards:
        sh.reset(src)
    lvl = 0
    while True:
        total = sum(sh.level_step(lvl) for sh in shards)
        if total == 0:
            return lvl + 1
        parts = [sh.next for sh in shards]
        for sh in shards:
            sh.place(parts)
        lvl += 1
