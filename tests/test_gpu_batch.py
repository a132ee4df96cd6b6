"""Batched traversals vs the oracle: multi-source BFS (bit frontier matrix)
and the multi-seed BFS over a block-diagonal batch of small graphs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def oracle_levels(orc, csr, srcs):
    return np.stack([orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, int(s))[0] for s in srcs], axis=1)


@pytest.mark.parametrize("k", [1, 5, 32, 64, 100, 256, 1024])
def test_msbfs_matches_per_source_bfs(gbo, orc, gpu, k):
    rng = np.random.default_rng(k)
    for csr in (gbo.gen_rmat(12, 16, seed=0), gbo.gen_er(1000, 0.02002, 0), gbo.gen_king_mesh(33)):
        g = gbo.Graph.from_csr(csr, 32)
        srcs = rng.integers(0, csr.nrows, k).astype(np.int32)
        lv, depth = g.msbfs(srcs)
        want = oracle_levels(orc, csr, srcs)
        assert np.array_equal(lv, want), (csr.nrows, k)
        assert depth == int(want.max()) + 1


@pytest.mark.parametrize("k", [1, 64, 100, 256, 1024])
def test_msbfs_seed_push_on_symmetric_graphs(gbo, orc, gpu, k):
    """On symmetric graphs whose levels all pull, level 0 pushes from the
    sources (hubs' tails split over warps, isolated sources, duplicates);
    every level matches one oracle BFS per source."""
    rng = np.random.default_rng(300 + k)
    e = rng.integers(0, 2000, (2, 12000)).astype(np.int32)
    island = gbo.csr_from_edges(e[0], e[1], 3000, True, True)  # 2000..2999 isolated
    hub = np.repeat(np.arange(3, dtype=np.int32), 19997)  # three hubs joined to every vertex
    leaves = np.tile(np.arange(3, 20000, dtype=np.int32), 3)
    star = gbo.csr_from_edges(hub, leaves, 20000, True, True)
    for csr in (gbo.gen_rmat(12, 16, seed=0), island, star):
        g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_SYMMETRIC)
        srcs = rng.integers(0, csr.nrows, k).astype(np.int32)
        srcs[0] = 0 if csr is not island else 2500  # a hub, or an isolated vertex
        if k > 1:
            srcs[-1] = srcs[0]
        want = oracle_levels(orc, csr, srcs)
        # 0: every level pulls after the seed push; the others push the
        # levels below the threshold over the slices (every level at 2^31-1)
        for push in (0, 4096, 2**31 - 1):
            g.set_bfs_direction(True, push)
            lv, depth = g.msbfs(srcs)
            assert np.array_equal(lv, want), (csr.nrows, k, push)
            assert depth == int(want.max()) + 1
            if push == 0:
                assert len(g.last_run()["step_ms"]) == depth
        g.free()


def test_msbfs_split_rows_and_duplicates(gbo, orc, gpu):
    # a hub vertex makes block row 0 long enough to be split across warps
    n = 20000
    src = np.zeros(n - 1, np.int32)
    dst = np.arange(1, n, dtype=np.int32)
    rng = np.random.default_rng(1)
    src = np.concatenate([src, rng.integers(0, n, 30000)]).astype(np.int32)
    dst = np.concatenate([dst, rng.integers(0, n, 30000)]).astype(np.int32)
    csr = gbo.csr_from_edges(src, dst, n, True, True)
    g = gbo.Graph.from_csr(csr, 32)
    assert g.info().nsplit_rows > 0
    srcs = np.array([5, 5, 0, 19999, 123] * 13, np.int32)  # duplicates allowed
    lv, _ = g.msbfs(srcs)
    assert np.array_equal(lv, oracle_levels(orc, csr, srcs))


@pytest.mark.parametrize("push", [0, 64, 2**31 - 1])
@pytest.mark.parametrize("k", [1, 5, 32, 33, 64])
def test_msbfs_push_levels_on_symmetric_graphs(gbo, orc, gpu, k, push):
    """On symmetric graphs with k <= 64 levels may push (frontier rows
    scattered to the neighbours): never (0), below 64 new (vertex, source)
    pairs, or always (2^31 - 1) -- the levels are the per-source BFS levels
    every time."""
    rng = np.random.default_rng(100 + k)
    # vertices 2000..2999 of the last graph have no edges (sources there too)
    e = rng.integers(0, 2000, (2, 12000)).astype(np.int32)
    island = gbo.csr_from_edges(e[0], e[1], 3000, True, True)
    graphs = (gbo.gen_rmat(12, 16, seed=0), gbo.gen_er(1000, 0.02002, 0), gbo.gen_king_mesh(33), island)
    for csr in graphs:
        g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_SYMMETRIC)
        g.set_bfs_direction(True, push)
        srcs = rng.integers(0, csr.nrows, k).astype(np.int32)
        if csr is island:
            srcs[0] = 2500
            srcs[-1] = srcs[0] if k > 1 else srcs[-1]  # a duplicate
        lv, depth = g.msbfs(srcs)
        want = oracle_levels(orc, csr, srcs)
        assert np.array_equal(lv, want), (csr.nrows, k, push)
        assert depth == int(want.max()) + 1
        # a second call on the same handle (captured graph reused)
        lv2, _ = g.msbfs(srcs)
        assert np.array_equal(lv2, want)
        g.free()


def test_msbfs_push_levels_split_rows(gbo, orc, gpu):
    n = 20000
    src = np.zeros(n - 1, np.int32)
    dst = np.arange(1, n, dtype=np.int32)
    rng = np.random.default_rng(2)
    src = np.concatenate([src, rng.integers(0, n, 30000)]).astype(np.int32)
    dst = np.concatenate([dst, rng.integers(0, n, 30000)]).astype(np.int32)
    csr = gbo.csr_from_edges(src, dst, n, True, True)
    g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_SYMMETRIC)
    assert g.info().nsplit_rows > 0
    srcs = np.array([5, 5, 0, 19999, 123] * 12 + [7, 8], np.int32)
    want = oracle_levels(orc, csr, srcs)
    for push in (64, 2**31 - 1, 0, -1, 64):  # the mode may change between calls
        g.set_bfs_direction(True, push)
        lv, _ = g.msbfs(srcs)
        assert np.array_equal(lv, want), push


def test_msbfs_push_covers_every_work_item(gbo, orc, gpu):
    """More work items than block rows (hub block row split into pieces) at a
    block-row count that fills whole blocks: every item must be pushed."""
    n = 32768  # 1024 block rows = 128 blocks of 8 warps
    hubs = np.repeat(np.arange(10, dtype=np.int32), n - 10)
    leaves = np.tile(np.arange(10, n, dtype=np.int32), 10)
    rng = np.random.default_rng(5)
    src = np.concatenate([hubs, rng.integers(0, n, 20000)]).astype(np.int32)
    dst = np.concatenate([leaves, rng.integers(0, n, 20000)]).astype(np.int32)
    csr = gbo.csr_from_edges(src, dst, n, True, True)
    g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_SYMMETRIC)
    assert g.info().nsplit_rows > 0 and g.info().nitems > 1024
    srcs = rng.integers(0, n, 64).astype(np.int32)
    want = oracle_levels(orc, csr, srcs)
    for push in (2**31 - 1, 4096, 0):
        g.set_bfs_direction(True, push)
        lv, _ = g.msbfs(srcs)
        assert np.array_equal(lv, want), push
    g.free()


def test_msbfs_rejects_other_tiles(gbo, gpu):
    g = gbo.Graph.from_csr(gbo.gen_er(200, 0.05, 1), 16)
    with pytest.raises(gbo.GboError) as e:
        g.msbfs([0, 1])
    assert e.value.status == gbo.GBO_ERR_UNSUPPORTED


@pytest.mark.parametrize("b", [4, 8, 32])
def test_batch_of_small_graphs_one_traversal(gbo, orc, gpu, b):
    csr, off = gbo.gen_er_batch(300, 32, 4096, 8.0, seed=7)
    seeds = off[:-1].copy()  # vertex 0 of every graph
    g = gbo.Graph.from_csr(csr, b)
    lv, _ = g.bfs_multi(seeds)
    for i in range(0, 300, 7):
        a, e = off[i], off[i + 1]
        sub_rp = csr.rowptr[a:e + 1] - csr.rowptr[a]
        sub_ci = csr.colind[csr.rowptr[a]:csr.rowptr[e]] - a
        want, _ = orc.bfs_csr(sub_rp, sub_ci, e - a, 0)
        assert np.array_equal(lv[a:e], want), i
    # whole batch against a multi-seed CPU BFS: per-graph levels never mix
    ref = np.full(csr.nrows, -1, np.int64)
    for i in range(300):
        a, e = off[i], off[i + 1]
        sub_rp = csr.rowptr[a:e + 1] - csr.rowptr[a]
        sub_ci = csr.colind[csr.rowptr[a]:csr.rowptr[e]] - a
        ref[a:e] = orc.bfs_csr(sub_rp, sub_ci, e - a, 0)[0]
    assert np.array_equal(lv, ref)
