"""B2SR packing on the GPU vs the oracle: byte-exact tiles, every tile width
and layout, the raw (caller-owned buffer) entry points and the error paths."""
import numpy as np
import pytest

from gpu_cases import cases

pytestmark = pytest.mark.gpu
WIDTHS = [4, 8, 16, 32, 64]


@pytest.fixture(scope="module")
def graphs(gbo):
    return cases(gbo)


@pytest.mark.parametrize("b", WIDTHS)
@pytest.mark.parametrize("layout", [0, 1])
def test_graph_pack_matches_oracle(gbo, orc, gpu, graphs, b, layout):
    for name, csr in graphs.items():
        flags = gbo.FLAG_LAYOUT_COL if layout else 0
        g = gbo.Graph.from_csr(csr, b, flags)
        rp, ci, w = g.b2sr()
        ref = orc.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, b, layout)
        assert np.array_equal(rp, ref.rowptr), (name, b)
        assert np.array_equal(ci, ref.colind), (name, b)
        assert np.array_equal(w, ref.narrow()), (name, b)
        inf = g.info()
        assert inf.nblocks == ref.nblk and inf.nblockrows == ref.nbr
        # out-degrees = column counts of the packed matrix
        assert np.array_equal(g.outdeg(), np.bincount(csr.colind, minlength=csr.ncols))


@pytest.mark.parametrize("b", WIDTHS)
def test_raw_pack_entry_points(gbo, orc, gpu, graphs, b):
    csr = graphs["rmat14"]
    drp = gbo.DeviceBuffer.from_numpy(csr.rowptr)
    dci = gbo.DeviceBuffer.from_numpy(csr.colind)
    for layout in (0, 1):
        brp, bci, val, nblk = gbo.b2sr_pack_raw(drp, dci, csr.nrows, csr.ncols, csr.nnz, b, layout)
        ref = orc.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, b, layout)
        assert nblk == ref.nblk
        assert np.array_equal(brp.to_numpy(np.int32), ref.rowptr)
        assert np.array_equal(bci.to_numpy(np.int32, nblk), ref.colind)
        assert np.array_equal(val.to_numpy(gbo.WORD_DTYPE[b], nblk * b), ref.narrow())


def test_transpose_and_lower_flags(gbo, orc, gpu, graphs):
    csr = graphs["ragged1001"]
    t = csr.transpose()
    low = graphs["rmat12"].tril()
    for b in (8, 32):
        g = gbo.Graph.from_csr(csr, b, gbo.FLAG_TRANSPOSE)
        rp, ci, w = g.b2sr()
        ref = orc.pack(t.rowptr, t.colind, t.nrows, t.ncols, b)
        assert np.array_equal(rp, ref.rowptr) and np.array_equal(ci, ref.colind)
        assert np.array_equal(w, ref.narrow())
        # PageRank degrees of P = A^T are A's row lengths
        assert np.array_equal(g.outdeg(), np.diff(csr.rowptr))
        gl = gbo.Graph.from_csr(graphs["rmat12"], b, gbo.FLAG_LOWER)
        rp, ci, w = gl.b2sr()
        ref = orc.pack(low.rowptr, low.colind, low.nrows, low.ncols, b)
        assert np.array_equal(ci, ref.colind) and np.array_equal(w, ref.narrow())


def test_duplicates_and_unsorted_and_bounds(gbo, orc, gpu):
    # duplicates (mmio_data keeps them) pack to the same bits
    rp = np.array([0, 3, 4], np.int32)
    ci = np.array([1, 1, 5, 0], np.int32)
    csr = gbo.Csr(rp, ci, 2, 8)
    g = gbo.Graph.from_csr(csr, 4)
    ref = orc.pack(rp, ci, 2, 8, 4)
    assert np.array_equal(g.b2sr()[2], ref.narrow())
    bad = gbo.Csr(np.array([0, 2], np.int32), np.array([5, 1], np.int32), 1, 8)
    with pytest.raises(gbo.GboError) as e:
        gbo.Graph.from_csr(bad, 4)
    assert e.value.status == gbo.GBO_ERR_UNSORTED
    oob = gbo.Csr(np.array([0, 2], np.int32), np.array([1, 9], np.int32), 1, 8)
    with pytest.raises(gbo.GboError) as e:
        gbo.Graph.from_csr(oob, 4)
    assert e.value.status == gbo.GBO_ERR_BOUNDS
    with pytest.raises(gbo.GboError) as e:
        gbo.Graph.from_csr(csr, 12)
    assert e.value.status == gbo.GBO_ERR_INVALID


def test_empty_graph(gbo, gpu):
    csr = gbo.Csr(np.zeros(6, np.int32), np.zeros(0, np.int32), 5, 5)
    for b in WIDTHS:
        g = gbo.Graph.from_csr(csr, b)
        assert g.info().nblocks == 0
        lv, depth = g.bfs(2)
        assert list(lv) == [-1, -1, 0, -1, -1] and depth == 1


@pytest.mark.parametrize("b", WIDTHS)
def test_vector_pack(gbo, orc, gpu, b):
    rng = np.random.default_rng(b)
    for n in (1, 31, 32, 33, 1000, 4097):
        x = (rng.random(n) < 0.5).astype(np.int32)
        ref = orc.pack_vector(x, b).astype(gbo.WORD_DTYPE[b])
        for kind, arr in (("f32", x.astype(np.float32)), ("i32", x)):
            dx = gbo.DeviceBuffer.from_numpy(arr)
            bits = gbo.pack_vector(dx, n, b, kind)
            got = bits.to_numpy(gbo.WORD_DTYPE[b], len(ref))
            assert np.array_equal(got, ref), (n, kind)
        assert np.array_equal(gbo.bits_from_numpy(x, b), ref)
        out = gbo.DeviceBuffer(4 * n)
        gbo.check(gbo.lib().gbo_unpack_vector(bits.ptr, n, b, out.ptr, None))
        assert np.array_equal(out.to_numpy(np.int32, n), x)
