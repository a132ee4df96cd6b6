"""Graph algorithms on the GPU vs the oracle: BFS levels, unit SSSP, CC labels
and triangle counts bit-exact; PageRank / PPR / PPR gradient within 1e-5
relative L1 of fp64."""
import numpy as np
import pytest

from conftest import sha
from gpu_cases import cases

pytestmark = pytest.mark.gpu
WIDTHS = [4, 8, 16, 32, 64]
INF = 2147483647


@pytest.fixture(scope="module")
def graphs(gbo):
    return cases(gbo)


def rel_l1(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).sum() / max(1e-300, np.abs(b).sum()))


@pytest.mark.parametrize("b", WIDTHS)
def test_bfs_and_sssp(gbo, orc, gpu, graphs, b):
    for name, csr in graphs.items():
        g = gbo.Graph.from_csr(csr, b)
        for src in (0, csr.nrows // 2, csr.nrows - 1):
            lv_ref, d_ref = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, src)
            lv, depth = g.bfs(src)
            assert np.array_equal(lv, lv_ref), (name, b, src)
            assert depth == d_ref
            dist, _ = g.sssp(src)
            assert np.array_equal(dist, np.where(lv_ref < 0, INF, lv_ref).astype(np.uint32)), (name, b)


def test_bfs_golden(gbo, gpu, golden):
    for key, csr in (("er1000", gbo.gen_er(1000, 0.02002, 0)), ("rmat12", gbo.gen_rmat(12, 16, seed=0)),
                     ("mesh33", gbo.gen_king_mesh(33))):
        g = gbo.Graph.from_csr(csr, 32)
        lv, depth = g.bfs(0)
        assert sha(lv) == golden[key]["bfs_levels_sha"] and depth == golden[key]["bfs_depth"]
        st = g.last_run()  # per-level times from device clock stamps at each level's end
        assert st["iterations"] == depth and len(st["step_ms"]) == depth
        # the cooperative loop launches 2 kernels (init, loop), the loop graph
        # 2 or 3 per level after init and loop start
        assert all(ms >= 0 for ms in st["step_ms"]) and st["kernel_launches"] in (2, 2 + 2 * depth, 2 + 3 * depth)


def test_bfs_transpose_directed(gbo, orc, gpu, graphs):
    """Directed graph: the reference packs the CSC so BFS follows A's edges."""
    a = graphs["ragged1001"]
    at = a.transpose()
    g = gbo.Graph.from_csr(a, 32, gbo.FLAG_TRANSPOSE)
    lv, _ = g.bfs(3)
    ref, _ = orc.bfs_csr(at.rowptr, at.colind, at.nrows, 3)
    assert np.array_equal(lv, ref)


@pytest.mark.parametrize("b", WIDTHS)
def test_cc_min_label(gbo, orc, gpu, graphs, b):
    for name, csr in graphs.items():
        if name == "ragged1001":
            continue  # CC needs a symmetric matrix
        g = gbo.Graph.from_csr(csr, b)
        lab, _ = g.cc()
        want = orc.cc(csr.rowptr, csr.colind, csr.nrows)
        assert np.array_equal(lab, want), (name, b)
        assert orc.verify_cc(csr.rowptr, csr.colind, csr.nrows, lab)[0] == 0


def test_cc_disconnected(gbo, orc, gpu):
    rng = np.random.default_rng(9)
    n = 5000
    src = rng.integers(0, n, 2500)
    dst = rng.integers(0, n, 2500)
    csr = gbo.csr_from_edges(src, dst, n, True, True)
    for b in WIDTHS:
        lab, _ = gbo.Graph.from_csr(csr, b).cc()
        assert np.array_equal(lab, orc.cc(csr.rowptr, csr.colind, n))


@pytest.mark.parametrize("b", WIDTHS)
def test_triangle_count(gbo, orc, gpu, graphs, b):
    for name, csr in graphs.items():
        rows = np.repeat(np.arange(csr.nrows), np.diff(csr.rowptr))
        if name == "ragged1001" or np.any(rows == csr.colind):
            continue  # TC is defined on simple undirected graphs
        g = gbo.Graph.from_csr(csr, b, gbo.FLAG_LOWER)
        assert g.tc() == orc.tc_csr(csr.rowptr, csr.colind, csr.nrows), (name, b)


def test_triangle_count_tensor_core_path(gbo, orc, gpu, graphs):
    """b = 32 with GBO_FLAG_TC_MMA: dense mask tiles through the 1-bit MMA."""
    for name in ("mesh33", "rmat12", "er1000", "star20000"):
        csr = graphs[name]
        for extra in (0, gbo.FLAG_DEGREE_ORDER):
            g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_LOWER | gbo.FLAG_TC_MMA | extra)
            assert g.tc() == orc.tc_csr(csr.rowptr, csr.colind, csr.nrows), (name, extra)
    for side in (64, 257):
        m = gbo.gen_king_mesh(side)
        assert gbo.Graph.from_csr(m, 32, gbo.FLAG_LOWER | gbo.FLAG_TC_MMA).tc() == 4 * (side - 1) ** 2


def test_triangle_mesh_closed_form(gbo, gpu):
    for side in (2, 3, 64, 257):
        m = gbo.gen_king_mesh(side)
        for b in (8, 16, 32, 64):
            assert gbo.Graph.from_csr(m, b, gbo.FLAG_LOWER).tc() == 4 * (side - 1) ** 2


@pytest.mark.parametrize("b", WIDTHS)
def test_pagerank(gbo, orc, gpu, graphs, b):
    for name, csr in graphs.items():
        g = gbo.Graph.from_csr(csr, b)
        outdeg = np.bincount(csr.colind, minlength=csr.ncols).astype(np.int32)
        p, it = g.pagerank(0.85, 20, -1.0)
        assert it == 20
        p64, _ = orc.pagerank_f64(csr.rowptr, csr.colind, csr.nrows, outdeg, 0.85, 20, -1.0)
        assert rel_l1(p, p64) <= 1e-5, (name, b, rel_l1(p, p64))
        # tolerance mode stops like the reference loop (pr.cu:449)
        p2, it2 = g.pagerank(0.85, 1000, 1e-6)
        p64b, it64 = orc.pagerank_f64(csr.rowptr, csr.colind, csr.nrows, outdeg, 0.85, 1000, 1e-6)
        assert abs(it2 - it64) <= 1 and rel_l1(p2, p64b) <= 1e-5


@pytest.mark.parametrize("b", [8, 32, 64])
@pytest.mark.parametrize("sym", [False, True])
def test_ppr_forward_backward(gbo, orc, gpu, b, sym):
    """sym: the graph is flagged symmetric, so the adjoint gathers over P's
    rows instead of scattering with atomics."""
    csr = gbo.gen_rmat(12, 16, seed=1)
    n = csr.nrows
    outdeg = np.bincount(csr.colind, minlength=n).astype(np.int32)
    rng = np.random.default_rng(4)
    v = np.zeros(n)
    idx = rng.choice(n, max(1, n // 100), replace=False)
    v[idx] = rng.dirichlet(np.ones(len(idx)))
    w = rng.standard_normal(n)
    g = gbo.Graph.from_csr(csr, b, gbo.FLAG_SYMMETRIC if sym else 0)
    p, _ = g.ppr_forward(v.astype(np.float32), 0.85, 1e-7, 1000)
    p64, _ = orc.ppr_f64(csr.rowptr, csr.colind, n, outdeg, v, 0.85, 1e-13)
    assert rel_l1(p, p64) <= 1e-5
    grad, _ = g.ppr_backward(w.astype(np.float32), 0.85, 1e-7, 1000)
    g64, _ = orc.ppr_adjoint_f64(csr.rowptr, csr.colind, n, outdeg, w, 0.85, 1e-13)
    assert rel_l1(grad, g64) <= 1e-5
    # central finite differences of L = w . p(v) through the GPU forward pass
    for _ in range(8):
        d = np.zeros(n)
        d[idx] = rng.standard_normal(len(idx))
        pp, _ = g.ppr_forward((v + 1e-3 * d).astype(np.float32), 0.85, 1e-9, 2000)
        pm, _ = g.ppr_forward((v - 1e-3 * d).astype(np.float32), 0.85, 1e-9, 2000)
        fd = (w @ pp.astype(np.float64) - w @ pm.astype(np.float64)) / 2e-3
        assert abs(fd - grad @ d) <= 2e-3 * max(1.0, abs(fd)) + 1e-4


@pytest.mark.parametrize("b", WIDTHS)
def test_bfs_direction_optimizing(gbo, orc, gpu, graphs, b):
    """Symmetric graphs may take top-down (push) steps: same levels."""
    for name, csr in graphs.items():
        if name == "ragged1001":
            continue  # not symmetric
        g = gbo.Graph.from_csr(csr, b, gbo.FLAG_SYMMETRIC)
        for src in (0, csr.nrows // 3, csr.nrows - 1):
            lv, depth = g.bfs(src)
            want, d = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, src)
            assert np.array_equal(lv, want), (name, b, src)
            assert depth == d
        # many seeds at once (block-diagonal batches) start in push mode too
        seeds = np.arange(0, csr.nrows, max(1, csr.nrows // 7), dtype=np.int32)
        lv, _ = g.bfs_multi(seeds)
        ref = np.full(csr.nrows, -1, np.int64)
        for s in seeds:
            x, _ = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, int(s))
            ref = np.where((ref < 0) | ((x >= 0) & (x < ref)), x, ref)
        assert np.array_equal(lv, ref), (name, b)


@pytest.mark.parametrize("b", WIDTHS)
def test_bfs_push_every_level(gbo, orc, gpu, graphs, b):
    """Threshold above n: every level is a top-down step (atomics into the
    next frontier), including the dense middle levels."""
    for name in ("rmat14", "mesh33", "star20000", "er1000", "latehub"):
        csr = graphs[name]
        g = gbo.Graph.from_csr(csr, b)
        g.set_bfs_direction(True, csr.nrows + 1)
        for src in (1, csr.nrows - 2):
            lv, depth = g.bfs(src)
            want, d = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, src)
            assert np.array_equal(lv, want) and depth == d, (name, b, src)
        g.set_bfs_direction(False)
        lv, _ = g.bfs(1)
        assert np.array_equal(lv, orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, 1)[0])


def test_bfs_cooperative_loop(gbo, orc, gpu, graphs):
    """The level loop as one cooperative launch (b = 32 ROW) gives the levels
    of the loop-graph form and of the oracle: pull-only, direction-optimising
    and every level pushed, single and many seeds, SSSP, and grids from one
    block to the device's limit."""
    cs = dict(graphs)
    cs["rmat18"] = gbo.gen_rmat(18, 16, seed=7)
    for name, csr in cs.items():
        sym = name != "ragged1001"
        g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_SYMMETRIC if sym else 0)
        srcs = (0, csr.nrows // 2, csr.nrows - 1)
        for thr in ((-1, csr.nrows + 1, 0) if sym else (0,)):
            g.set_bfs_direction(sym and thr != 0, thr)
            for blocks in (0, 1, 7, 1 << 20):
                g.set_bfs_loop(gbo.BFS_LOOP_COOP, blocks)
                for src in srcs:
                    want, d = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, src)
                    lv, depth = g.bfs(src)
                    assert np.array_equal(lv, want) and depth == d, (name, thr, blocks, src)
                    st = g.last_run()
                    assert st["iterations"] == depth and len(st["step_ms"]) == min(depth, 4096)
                    assert st["kernel_launches"] == 2
            g.set_bfs_loop(gbo.BFS_LOOP_GRAPH)
            lv, depth = g.bfs(srcs[1])
            assert np.array_equal(lv, orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, srcs[1])[0]), (name, thr)
        g.set_bfs_loop(gbo.BFS_LOOP_COOP)
        dist, _ = g.sssp(1 % csr.nrows)
        want, _ = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, 1 % csr.nrows)
        assert np.array_equal(dist, np.where(want < 0, INF, want).astype(np.uint32)), name
        seeds = np.arange(0, csr.nrows, max(1, csr.nrows // 5), dtype=np.int32)
        lv, _ = g.bfs_multi(seeds)
        ref = np.full(csr.nrows, -1, np.int64)
        for s in seeds:
            x, _ = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, int(s))
            ref = np.where((ref < 0) | ((x >= 0) & (x < ref)), x, ref)
        assert np.array_equal(lv, ref), name
        g.free()


def test_bfs_cooperative_loop_rejected(gbo, gpu, graphs):
    g = gbo.Graph.from_csr(graphs["er1000"], 8)
    with pytest.raises(gbo.GboError) as e:
        g.set_bfs_loop(gbo.BFS_LOOP_COOP)
    assert e.value.status == gbo.GBO_ERR_UNSUPPORTED
    with pytest.raises(gbo.GboError):
        g.set_bfs_loop(7)
    g.set_bfs_loop(gbo.BFS_LOOP_GRAPH)
    g.free()


@pytest.mark.parametrize("b", WIDTHS)
def test_bfs_col_layout(gbo, orc, gpu, graphs, b):
    """BFS and SSSP on column-word tiles: pull-only, direction-optimising,
    every level pushed, and many seeds, all equal to the oracle."""
    for name, csr in graphs.items():
        sym = name != "ragged1001"
        g = gbo.Graph.from_csr(csr, b, gbo.FLAG_LAYOUT_COL | (gbo.FLAG_SYMMETRIC if sym else 0))
        for thr in ((-1, csr.nrows + 1, 0) if sym else (0,)):
            g.set_bfs_direction(sym and thr != 0, thr)
            for src in (0, csr.nrows // 2, csr.nrows - 1):
                want, d = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, src)
                lv, depth = g.bfs(src)
                assert np.array_equal(lv, want) and depth == d, (name, b, thr, src)
        dist, _ = g.sssp(1 % csr.nrows)
        want, _ = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, 1 % csr.nrows)
        assert np.array_equal(dist, np.where(want < 0, INF, want).astype(np.uint32)), (name, b)
        seeds = np.arange(0, csr.nrows, max(1, csr.nrows // 5), dtype=np.int32)
        lv, _ = g.bfs_multi(seeds)
        ref = np.full(csr.nrows, -1, np.int64)
        for s in seeds:
            x, _ = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, int(s))
            ref = np.where((ref < 0) | ((x >= 0) & (x < ref)), x, ref)
        assert np.array_equal(lv, ref), (name, b)


@pytest.mark.parametrize("b", [8, 16, 32, 64])
def test_degree_order(gbo, orc, gpu, graphs, b):
    """Relabelling by descending degree: the triangle count is unchanged and
    BFS levels are the original ones under the returned labels."""
    for name in ("rmat12", "rmat14", "er1000", "mesh33", "star20000"):
        csr = graphs[name]
        g = gbo.Graph.from_csr(csr, b, gbo.FLAG_LOWER | gbo.FLAG_DEGREE_ORDER)
        assert g.tc() == orc.tc_csr(csr.rowptr, csr.colind, csr.nrows), (name, b)
        perm = g.permutation()
        assert np.array_equal(np.sort(perm), np.arange(csr.nrows))
        deg = np.diff(csr.rowptr)
        assert np.all(np.diff(deg[np.argsort(perm)]) <= 0)  # labels by descending degree
        h = gbo.Graph.from_csr(csr, b, gbo.FLAG_DEGREE_ORDER | gbo.FLAG_SYMMETRIC)
        lv, _ = h.bfs(int(perm[3]))
        want, _ = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, 3)
        assert np.array_equal(lv[perm], want), (name, b)
    assert gbo.Graph.from_csr(graphs["mesh33"], 8).permutation() is None
