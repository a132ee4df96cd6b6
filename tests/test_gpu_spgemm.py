"""Unmasked binary products on B2SR against the oracle: the total of A B
(bmm*_sparse, bsrbmm/bsrbmm.cu:244-555) at every tile width and layout, and
the sparse-output product C = A B (bsrbmm/bsrbmm.cu:1273-1373) entry for
entry, including L L^T (benchmark-bsrbmm.cu's check) on a graph whose tile
pairs span several processing ranges."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rect(gbo, n, m, p, seed):
    rng = np.random.default_rng(seed)
    d = rng.random((n, m)) < p
    rowptr = np.concatenate([[0], np.cumsum(d.sum(1))]).astype(np.int32)
    return gbo.Csr(rowptr, np.nonzero(d)[1].astype(np.int32), n, m)


def _cases(gbo):
    low = gbo.gen_rmat(10, 8, seed=7).tril()
    mesh = gbo.gen_king_mesh(40).tril()
    return [("rmat10 L L^T", low, low.transpose()),
            ("mesh40 L L^T", mesh, mesh.transpose()),
            ("rectangular", _rect(gbo, 300, 170, 0.04, 1), _rect(gbo, 170, 410, 0.06, 2))]


def test_spgemm_matches_oracle(gbo, orc, gpu):
    for name, a, b in _cases(gbo):
        ga = gbo.Graph.from_csr(a, 32)
        gb = gbo.Graph.from_csr(b, 32, gbo.FLAG_LAYOUT_COL)
        rp, ci, v = ga.spgemm(gb)
        wrp, wci, wv = orc.spgemm_csr(a.rowptr, a.colind, a.nrows, b.rowptr, b.colind, b.ncols)
        assert np.array_equal(rp, wrp), name
        assert np.array_equal(ci, wci) and np.array_equal(v, wv), name
        assert ga.bmm_sum(gb) == int(wv.sum()), name
        ga.free()
        gb.free()


@pytest.mark.parametrize("b", [4, 8, 16, 32, 64])
def test_bmm_sum_every_width_and_layout(gbo, orc, gpu, b):
    for name, a, bm in _cases(gbo):
        want = int(orc.spgemm_csr(a.rowptr, a.colind, a.nrows, bm.rowptr, bm.colind, bm.ncols)[2].sum())
        assert want == orc.bmm_sum_b2sr(orc.pack(a.rowptr, a.colind, a.nrows, a.ncols, b),
                                        orc.pack(bm.rowptr, bm.colind, bm.nrows, bm.ncols, b, layout=1))
        for fa in (0, gbo.FLAG_LAYOUT_COL):
            for fb in (0, gbo.FLAG_LAYOUT_COL):
                ga = gbo.Graph.from_csr(a, b, fa)
                gb = gbo.Graph.from_csr(bm, b, fb)
                assert ga.bmm_sum(gb) == want, (name, fa, fb)
                ga.free()
                gb.free()


def test_spgemm_several_pair_ranges(gbo, orc, gpu):
    # ER n = 12000, p = 0.003: every 32x32 tile is occupied, 48 M tile pairs
    # (more than one processing range of 2^25 pairs), 14.8 M entries of A^2
    g = gbo.gen_er(12000, 0.003, 9)
    ga = gbo.Graph.from_csr(g, 32)
    gb = gbo.Graph.from_csr(g, 32, gbo.FLAG_LAYOUT_COL)
    rp, ci, v = ga.spgemm(gb)
    wrp, wci, wv = orc.spgemm_csr(g.rowptr, g.colind, g.nrows, g.rowptr, g.colind, g.ncols)
    assert np.array_equal(rp, wrp) and np.array_equal(ci, wci) and np.array_equal(v, wv)
    assert ga.bmm_sum(gb) == int(wv.sum())


def test_spgemm_rejects_other_layouts(gbo, gpu):
    a = _rect(gbo, 64, 64, 0.1, 3)
    ga = gbo.Graph.from_csr(a, 32)
    with pytest.raises(gbo.GboError) as e:
        ga.spgemm(ga)  # B must carry column words
    assert e.value.status == gbo.GBO_ERR_UNSUPPORTED
    g16 = gbo.Graph.from_csr(a, 16)
    with pytest.raises(gbo.GboError):
        g16.bmm_sum(ga)  # tile widths differ


def test_products_of_empty_matrices(gbo, gpu):
    empty = gbo.Csr(np.zeros(65, np.int32), np.zeros(0, np.int32), 64, 64)
    a = _rect(gbo, 64, 64, 0.1, 4)
    for x, y in ((empty, a), (a, empty), (empty, empty)):
        gx = gbo.Graph.from_csr(x, 32)
        gy = gbo.Graph.from_csr(y, 32, gbo.FLAG_LAYOUT_COL)
        rp, ci, v = gx.spgemm(gy)
        assert rp.shape == (65,) and not rp.any() and len(ci) == 0 and len(v) == 0
        assert gx.bmm_sum(gy) == 0
        gx.free()
        gy.free()
