"""B2SR cache file: a saved and reloaded graph has the same B2SR arrays and
gives the same results; malformed files are rejected with GBO_ERR_IO."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("b", [4, 8, 16, 32, 64])
def test_save_load_roundtrip(gbo, gpu, tmp_path, b):
    csr = gbo.gen_rmat(11, 16, seed=3)
    g = gbo.Graph.from_csr(csr, b, gbo.FLAG_SYMMETRIC)
    path = str(tmp_path / f"g{b}.b2sr")
    g.save(path)
    h = gbo.Graph.load(path)
    for a0, a1 in zip(g.b2sr(), h.b2sr()):
        assert np.array_equal(a0, a1)
    assert np.array_equal(g.outdeg(), h.outdeg())
    i0, i1 = g.info(), h.info()
    assert (i0.nrows, i0.ncols, i0.nblocks, i0.nnz, i0.nitems) == (i1.nrows, i1.ncols, i1.nblocks, i1.nnz, i1.nitems)
    lv0, d0 = g.bfs(5)
    lv1, d1 = h.bfs(5)
    assert d0 == d1 and np.array_equal(lv0, lv1)
    p0, _ = g.pagerank(0.85, 20)
    p1, _ = h.pagerank(0.85, 20)
    assert np.array_equal(p0, p1)
    g.free()
    h.free()


def test_save_load_lower_and_degree_order(gbo, gpu, tmp_path):
    csr = gbo.gen_rmat(11, 16, seed=4)
    g = gbo.Graph.from_csr(csr, 16, gbo.FLAG_LOWER | gbo.FLAG_DEGREE_ORDER)
    path = str(tmp_path / "lower.b2sr")
    g.save(path)
    h = gbo.Graph.load(path)
    assert g.tc() == h.tc()
    assert np.array_equal(g.permutation(), h.permutation())
    g.free()
    h.free()


def test_load_rejects_malformed_files(gbo, gpu, tmp_path):
    csr = gbo.gen_rmat(10, 8, seed=5)
    g = gbo.Graph.from_csr(csr, 32)
    path = tmp_path / "g.b2sr"
    g.save(str(path))
    raw = path.read_bytes()
    bad = tmp_path / "bad.b2sr"
    for blob in (raw[:-7],                 # truncated tile words
                 b"XXXXXXXX" + raw[8:],     # wrong magic
                 raw[:64] + (1).to_bytes(4, "little") + raw[68:]):  # first block-row offset not 0
        bad.write_bytes(blob)
        with pytest.raises(gbo.GboError) as e:
            gbo.Graph.load(str(bad))
        assert e.value.status == gbo.GBO_ERR_IO
    with pytest.raises(gbo.GboError) as e:
        gbo.Graph.load(str(tmp_path / "missing.b2sr"))
    assert e.value.status == gbo.GBO_ERR_IO
    g.free()


def test_save_load_empty_graph(gbo, gpu, tmp_path):
    empty = gbo.Csr(np.zeros(101, np.int32), np.zeros(0, np.int32), 100, 100)
    g = gbo.Graph.from_csr(empty, 32)
    path = str(tmp_path / "empty.b2sr")
    g.save(path)
    h = gbo.Graph.load(path)
    assert h.info().nblocks == 0 and h.info().nrows == 100
    lv, depth = h.bfs(3)
    assert lv[3] == 0 and (lv[np.arange(100) != 3] == -1).all()
    g.free()
    h.free()
