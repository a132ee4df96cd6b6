"""The benchmark's algorithmic-bytes model of a BFS pull step
(bench.bfs_level_bytes), which sets the roofline's `achieved`, against a
direct count over the tiles of a small graph (CPU only)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def block_structure(csr, b):
    """Block-row offsets and block-column indices of the B2SR tiles of a CSR."""
    nbr = (csr.nrows + b - 1) // b
    rows = np.repeat(np.arange(csr.nrows), np.diff(csr.rowptr))
    keys = np.unique((rows // b).astype(np.int64) * (1 << 32) + csr.colind // b)
    br, bc = keys >> 32, keys & 0xFFFFFFFF
    rowptr_b = np.zeros(nbr + 1, np.int64)
    np.add.at(rowptr_b, br + 1, 1)
    return np.cumsum(rowptr_b), bc.astype(np.int64)


def direct_bytes(csr, rowptr_b, colind_b, levels, b, layout):
    """Bytes of each pull step, counted tile by tile from the model's words."""
    n, nbr = csr.nrows, len(rowptr_b) - 1
    wb = max(1, b // 8)
    deg = np.diff(csr.rowptr)
    occ = b == 32 and layout == "row"
    out = []
    for L in range(int(levels.max()) + 1):
        unvisited = [(levels[v] == -1 or levels[v] > L) for v in range(n)]
        frontier = [levels[v] == L for v in range(n)]
        by = 4 * (nbr + 1) + 2 * wb * nbr
        by += 4 * int((levels == L + 1).sum())
        by += wb * sum(any(levels[v] == L + 1 for v in range(R * b, min(n, R * b + b))) for R in range(nbr))
        for R in range(nbr):
            rows = range(R * b, min(n, R * b + b))
            open_rows = [v for v in rows if unvisited[v] and deg[v] > 0]
            if not open_rows:
                continue
            for t in range(rowptr_b[R], rowptr_b[R + 1]):
                C = colind_b[t]
                cols = range(C * b, min(n, C * b + b))
                by += 4 * (2 if occ else 1)  # block-column index (+ occupancy word)
                fr = [u for u in cols if frontier[u]]
                if not fr:
                    continue
                if occ:  # non-empty row words of unvisited rows
                    for v in rows:
                        if not unvisited[v]:
                            continue
                        nb = csr.colind[csr.rowptr[v]:csr.rowptr[v + 1]]
                        if np.any((nb >= C * b) & (nb < C * b + b)):
                            by += wb
                elif layout == "col":
                    by += wb * len(fr)
                else:
                    by += wb * len(open_rows)
        out.append(by)
    return out


@pytest.mark.parametrize("b,layout", [(8, "row"), (32, "row"), (16, "col"), (32, "col")])
def test_bfs_level_bytes_matches_direct_count(gbo, orc, b, layout):
    csr = gbo.gen_rmat(9, 6, seed=4)
    levels, _ = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, 0)
    levels = np.asarray(levels, np.int64)
    rowptr_b, colind_b = block_structure(csr, b)
    live = np.diff(csr.rowptr) > 0
    got = bench.bfs_level_bytes(rowptr_b, colind_b, levels, csr.nrows, b, live, layout, csr)
    want = direct_bytes(csr, rowptr_b, colind_b, levels, b, layout)
    assert got == want


def test_cpu_baseline_single_thread_restores_threads(gbo, orc):
    csr = gbo.gen_rmat(10, 8, seed=1)
    before = orc.max_threads()
    bs = orc.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, 32)
    v1, t1 = bench.cpu_bfs_single(orc, bs, csr, 3)
    assert v1 > 0 and t1 > 0
    assert orc.max_threads() == before
    v, t, cores, lv, depth = bench.cpu_bfs(orc, bs, csr, 2)
    assert v > 0 and cores == before
    assert np.array_equal(lv, orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, 0)[0])


def test_bfs_level_bytes_rws_matches_direct_count(gbo, orc):
    """The row-word slice pull model against a row-by-row walk."""
    csr = gbo.gen_rmat(9, 6, seed=4)
    n = csr.nrows
    levels = np.asarray(orc.bfs_csr(csr.rowptr, csr.colind, n, 0)[0], np.int64)
    got = bench.bfs_level_bytes_rws(csr, levels, head=3)
    nbr = (n + 31) // 32
    want = []
    for L in range(int(levels.max()) + 1):
        by = 8 * nbr + 4 * int((levels == L + 1).sum())
        by += 8 * sum(any(levels[v] == L + 1 for v in range(R * 32, min(n, R * 32 + 32))) for R in range(nbr))
        for v in range(n):
            nb = csr.colind[csr.rowptr[v]:csr.rowptr[v + 1]]
            if len(nb) == 0 or not (levels[v] == -1 or levels[v] > L):
                continue
            blocks = sorted(set(int(c) // 32 for c in nb))
            seen = 0
            for C in blocks:
                seen += 1
                if any(levels[u] == L for u in nb if u // 32 == C):
                    break
            by += 8 * seen + (16 if seen > 3 else 0)
        want.append(by)
    assert got == want


def test_bfs_push_bytes_rws_matches_direct_count(gbo, orc):
    """The slice push model (cooperative loop) against a row-by-row walk."""
    csr = gbo.gen_rmat(9, 6, seed=4)
    n = csr.nrows
    levels = np.asarray(orc.bfs_csr(csr.rowptr, csr.colind, n, 0)[0], np.int64)
    nbr = (n + 31) // 32
    for head, long_tail in ((8, 64), (2, 3)):
        for L in range(int(levels.max()) + 1):
            got = bench.bfs_push_bytes_rws(csr, levels, L, head=head, long_tail=long_tail)
            by = 8 * nbr + 4 * int((levels == L + 1).sum())
            by += 8 * sum(any(levels[v] == L + 1 for v in range(R * 32, min(n, R * 32 + 32))) for R in range(nbr))
            for v in np.flatnonzero(levels == L):
                blocks = set(int(c) // 32 for c in csr.colind[csr.rowptr[v]:csr.rowptr[v + 1]])
                tail = max(0, len(blocks) - head)
                by += 16 + 8 * head + 8 * tail + (16 if tail > long_tail else 0)
            assert got == by, (head, L)


@pytest.mark.parametrize("slots", [32, 64, 256, 1024])
def test_warm_server_runs_one_batch_per_frontier_width(slots):
    """bench.warm_server submits batches of 1, 33, 65, ... queries, each
    collected before the next, so that a batch-mode server has run one batch
    at every frontier width (32, 64, ... slots columns) before a stream."""
    class FakeLib:
        def __init__(self):
            self.waited = []

        def gbo_server_wait(self, h, t, out, lat, it, timeout):
            self.waited.append(t)
            return 0

    class FakeGbo:
        def __init__(self):
            self._lib = FakeLib()

        def lib(self):
            return self._lib

        @staticmethod
        def check(st, what):
            assert st == 0, what

    class FakeServer:
        h = None

        def __init__(self):
            self.batches, self.next = [], 1

        def submit_bfs(self, src):
            self.batches[-1].append(self.next)
            self.next += 1
            return self.next - 1

    fg, srv = FakeGbo(), FakeServer()
    orig = srv.submit_bfs
    sizes = []

    def submit(src):
        if not sizes or len(fg.lib().waited) == sum(sizes):
            sizes.append(0)
            srv.batches.append([])
        sizes[-1] += 1
        return orig(src)

    srv.submit_bfs = submit
    bench.warm_server(fg, srv, 1000, slots, 0)
    widths = set()
    for m in sizes:
        w = 32
        while w < m:
            w *= 2
        widths.add(w)
    want, w = set(), 32
    while w <= slots:
        want.add(w)
        w *= 2
    assert widths == want, (sizes, widths)
    assert fg.lib().waited == list(range(1, sum(sizes) + 1))
