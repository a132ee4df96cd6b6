"""Pins the CPU oracle against known answers (tests/golden/golden.json, from
networkx/scipy) and closed forms, before it is trusted as the GPU checker."""
import numpy as np
import pytest

from conftest import ref_path, sha


def _graphs(gbo, golden):
    out = {"er1000": gbo.gen_er(1000, 0.02002, 0), "rmat12": gbo.gen_rmat(12, 16, seed=0)}
    for side in (2, 3, 8, 33):
        out[f"mesh{side}"] = gbo.gen_king_mesh(side)
    for key, rel in (("bsrbmv_test", "bsrbmv/test.mtx"), ("bsrbmm_test", "bsrbmm/test.mtx"),
                     ("G43", "bsrbmv/G43.mtx")):
        p = ref_path(rel)
        if p and f"{key}_readmtx" in golden:
            out[f"{key}_readmtx"] = gbo.read_mtx(p, gbo.MTX_READMTX, 0)
            out[f"{key}_mmio"] = gbo.read_mtx(p, gbo.MTX_MMIO, 0)
    return out


@pytest.fixture(scope="module")
def graphs(gbo, golden):
    return _graphs(gbo, golden)


def test_inputs_match_golden(graphs, golden):
    for k, csr in graphs.items():
        g = golden[k]
        assert csr.nrows == g["n"] and csr.nnz == g["nnz"], k
        assert sha(csr.rowptr) == g["rowptr_sha"] and sha(csr.colind) == g["colind_sha"], k


@pytest.mark.parametrize("b", [4, 8, 16, 32, 64])
def test_oracle_bmv_count_golden(graphs, golden, orc, b):
    for k, csr in graphs.items():
        g = golden[k]
        x = (np.random.default_rng(g["bmv_x_seed"]).random(csr.ncols) < 0.5).astype(np.int32)
        bs = orc.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, b)
        y = orc.bmv_count(bs, orc.pack_vector(x, b))
        if "mmio" not in k:  # duplicates would differ between bits and counts
            assert sha(y) == g["bmv_count_sha"], (k, b)
        assert int(y.sum()) <= g["bmv_count_sum"]


@pytest.mark.parametrize("b", [4, 32, 64])
def test_oracle_bfs_golden(graphs, golden, orc, b):
    for k, csr in graphs.items():
        g = golden[k]
        bs = orc.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, b)
        lv, depth = orc.bfs_b2sr(bs, g["bfs_src"])
        assert sha(lv) == g["bfs_levels_sha"], (k, b)
        assert depth == g["bfs_depth"]
        lv2, _ = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, g["bfs_src"])
        assert np.array_equal(lv, lv2)
        d, _ = orc.sssp_b2sr(bs, g["bfs_src"])
        assert np.array_equal(np.where(lv < 0, orc.INF, lv).astype(np.uint32), d)


def test_oracle_triangles_and_cc_golden(graphs, golden, orc):
    for k, csr in graphs.items():
        g = golden[k]
        if "triangles" not in g or "mmio" in k:
            continue
        assert orc.tc_csr(csr.rowptr, csr.colind, csr.nrows) == g["triangles"], k
        if "triangles_closed_form" in g:
            assert g["triangles"] == g["triangles_closed_form"]
            assert csr.nnz // 2 == g["edges_closed_form"]
        for b in (8, 32, 64):
            low = csr.tril()
            assert orc.tc_b2sr(orc.pack(low.rowptr, low.colind, low.nrows, low.ncols, b)) == g["triangles"]
        lab = orc.cc(csr.rowptr, csr.colind, csr.nrows)
        assert sha(lab) == g["cc_labels_sha"], k
        err, ncomp = orc.verify_cc(csr.rowptr, csr.colind, csr.nrows, lab)
        assert err == 0 and ncomp == g["components"]


def test_oracle_pagerank_golden(graphs, golden, orc):
    for k, csr in graphs.items():
        g = golden[k]
        outdeg = np.bincount(csr.colind, minlength=csr.ncols).astype(np.int32)
        p64, it = orc.pagerank_f64(csr.rowptr, csr.colind, csr.nrows, outdeg, 0.85, 20, -1.0)
        assert it == 20
        np.testing.assert_allclose(p64[:8], g["pr20"][: len(p64[:8])], rtol=1e-12, atol=1e-15)
        bs = orc.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, 32)
        p32, _ = orc.pagerank_b2sr_f32(bs, outdeg, 0.85, 20, -1.0)
        assert np.abs(p32 - p64).sum() / np.abs(p64).sum() < 1e-5, k


def test_oracle_mesh_big_closed_form(gbo, orc):
    m = gbo.gen_king_mesh(256)
    assert orc.tc_csr(m.rowptr, m.colind, m.nrows) == 4 * 255 ** 2
    lv, d = orc.bfs_csr(m.rowptr, m.colind, m.nrows, 0)
    r, c = np.divmod(np.arange(m.nrows), 256)
    assert np.array_equal(lv, np.maximum(r, c)) and d == 256


def test_oracle_layout_col_is_transposed_tiles(gbo, orc):
    csr = gbo.gen_rmat(10, 8, seed=3)
    for b in (4, 8, 16, 32, 64):
        row = orc.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, b, 0)
        col = orc.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, b, 1)
        assert np.array_equal(row.rowptr, col.rowptr) and np.array_equal(row.colind, col.colind)
        w = row.words.reshape(-1, b)
        bits = ((w[:, :, None] >> np.arange(b - 1, -1, -1, dtype=np.uint64)[None, None, :]) & 1)
        wt = (bits.transpose(0, 2, 1) * (np.uint64(1) << np.arange(b - 1, -1, -1, dtype=np.uint64))).sum(
            axis=2, dtype=np.uint64)
        assert np.array_equal(wt.reshape(-1), col.words)


def test_oracle_ppr_adjoint_matches_finite_difference(gbo, orc):
    csr = gbo.gen_rmat(9, 8, seed=5)
    n = csr.nrows
    outdeg = np.bincount(csr.colind, minlength=n).astype(np.int32)
    rng = np.random.default_rng(0)
    v = rng.dirichlet(np.ones(n))
    w = rng.standard_normal(n)
    grad, _ = orc.ppr_adjoint_f64(csr.rowptr, csr.colind, n, outdeg, w, 0.85, 1e-14)
    for _ in range(4):
        d = rng.standard_normal(n)
        pp, _ = orc.ppr_f64(csr.rowptr, csr.colind, n, outdeg, v + 1e-3 * d, 0.85, 1e-14)
        pm, _ = orc.ppr_f64(csr.rowptr, csr.colind, n, outdeg, v - 1e-3 * d, 0.85, 1e-14)
        fd = (w @ pp - w @ pm) / 2e-3
        assert abs(fd - grad @ d) <= 1e-6 * max(1.0, abs(fd))


def test_oracle_reference_fixture_readers(orc, gbo):
    for rel in ("bsrbmv/test.mtx", "bsrbmm/test.mtx", "bsrbmv/G43.mtx"):
        p = ref_path(rel)
        if not p:
            pytest.skip("reference checkout not mounted")
        for d in (0, 1, 2):
            nr, nc, rp, ci = orc.read_mtx_readmtx(p, d)
            c = gbo.read_mtx(p, gbo.MTX_READMTX, d)
            assert (c.nrows, c.ncols) == (nr, nc)
            assert np.array_equal(c.rowptr, rp) and np.array_equal(c.colind, ci)
        nr, nc, rp, ci = orc.read_mtx_mmio(p)
        c = gbo.read_mtx(p, gbo.MTX_MMIO, 0)
        assert np.array_equal(c.rowptr, rp) and np.array_equal(c.colind, ci)


def _rect_csr(n, m, p, seed):
    rng = np.random.default_rng(seed)
    d = rng.random((n, m)) < p
    rowptr = np.concatenate([[0], np.cumsum(d.sum(1))]).astype(np.int32)
    return rowptr, np.nonzero(d)[1].astype(np.int32), d


def test_oracle_spgemm_and_bmm_sum_vs_scipy(gbo, orc):
    """The oracle's sparse-output product and its tile-level total
    (bsrbmm/bsrbmm.cu:244-555, 1273-1373) against scipy's product."""
    import scipy.sparse as sp

    cases = []
    csr = gbo.gen_rmat(9, 8, seed=7)
    low = csr.tril()
    lt = low.transpose()
    cases.append((low.rowptr, low.colind, low.nrows, low.ncols, lt.rowptr, lt.colind, lt.ncols))
    arp, aci, _ = _rect_csr(150, 90, 0.05, 1)
    brp, bci, _ = _rect_csr(90, 200, 0.08, 2)
    cases.append((arp, aci, 150, 90, brp, bci, 200))
    for arp, aci, n, k, brp, bci, m in cases:
        A = sp.csr_matrix((np.ones(len(aci), np.int64), aci, arp), shape=(n, k))
        B = sp.csr_matrix((np.ones(len(bci), np.int64), bci, brp), shape=(k, m))
        Cm = (A @ B).tocsr()
        Cm.sort_indices()
        rp, ci, v = orc.spgemm_csr(arp, aci, n, brp, bci, m)
        assert np.array_equal(rp, Cm.indptr) and np.array_equal(ci, Cm.indices)
        assert np.array_equal(v, Cm.data)
        for b in (8, 32):
            a_t = orc.pack(arp, aci, n, k, b)
            b_t = orc.pack(brp, bci, k, m, b, layout=1)
            assert orc.bmm_sum_b2sr(a_t, b_t) == int(Cm.sum())
