"""gbo_bmv_count_noalloc (static device scratch, no allocation) against
the oracle's BMV count and gbo_bmv_count on the same packed graphs:
identical integer counts, two calls in a row with different vectors so that
stale scratch would show, and a hand-built B2SR whose row lengths put every
split-row case into the chunks.  The file is named to be collected last; it
also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
WIDTHS = [4, 8, 16, 32, 64]
ERR_UNSUPPORTED = 8


def _star_plus_rmat(gbo, n=100_000):
    """Vertex 0 adjacent to every vertex (block row 0 spans several chunks
    at every tile width) plus an R-MAT scale-14 graph on the low vertices."""
    r = gbo.gen_rmat(14, 16, seed=5)
    rows = np.repeat(np.arange(r.nrows, dtype=np.int32), np.diff(r.rowptr))
    src = np.concatenate([np.zeros(n - 1, np.int32), rows])
    dst = np.concatenate([np.arange(1, n, dtype=np.int32), r.colind.astype(np.int32)])
    return gbo.csr_from_edges(src, dst, n, True, True)


def _noalloc(gbo, g, dx, dy, out_type, accumulate):
    info = g.info()
    r, c, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
    gbo.check(gbo.lib().gbo_graph_b2sr(g.h, C.byref(r), C.byref(c), C.byref(v)), "graph_b2sr")
    return gbo.lib().gbo_bmv_count_noalloc(info.nrows, info.ncols, info.tile_bits, int(info.nblocks),
                                           r, c, v, dx.ptr, dy.ptr, out_type, int(accumulate), None)


@pytest.mark.parametrize("b", WIDTHS)
def test_noalloc_matches_bmv_count(gbo, orc, gpu, b):
    rng = np.random.default_rng(40 + b)
    for csr in (_star_plus_rmat(gbo), gbo.gen_rmat(12, 16, seed=2), gbo.gen_er(1001, 0.01, 3)):
        g = gbo.Graph.from_csr(csr, b)
        n = csr.nrows
        for call in range(2):  # two calls in a row, different x
            x = (rng.random(csr.ncols) < (0.5 if call == 0 else 0.2)).astype(np.int32)
            dx = gbo.DeviceBuffer.from_numpy(gbo.bits_from_numpy(x, b))
            want = gbo.DeviceBuffer(4 * n)
            g.bmv_count(dx, want)
            y = gbo.DeviceBuffer.from_numpy(np.full(n, -7, np.int32))  # overwritten
            gbo.check(_noalloc(gbo, g, dx, y, gbo.OUT_I32, False), "bmv_count_noalloc")
            ref = want.to_numpy(np.int32, n)
            got = y.to_numpy(np.int32, n)
            assert np.array_equal(got, ref), (b, n, call)
            if call == 0:  # and straight against the oracle's count on the CPU packing
                ob = orc.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, b)
                assert np.array_equal(got, orc.bmv_count(ob, orc.pack_vector(x, b))), (b, n)
            # float output accumulated onto a base, as gbo_bmv_count does
            base = rng.integers(0, 5, n).astype(np.float32)
            yf = gbo.DeviceBuffer.from_numpy(base)
            gbo.check(_noalloc(gbo, g, dx, yf, gbo.OUT_F32, True), "bmv_count_noalloc f32")
            assert np.array_equal(yf.to_numpy(np.float32, n), base + ref.astype(np.float32)), (b, call)
        g.free()


def test_noalloc_rejects_graphs_beyond_its_scratch(gbo, gpu):
    # 2^35 / b^2 tiles at most; checked before any pointer is used or launch made
    for b in WIDTHS:
        limit = min(2**35 // (b * b), 2**31 - 1)
        if limit >= 2**31 - 1:
            continue
        st = gbo.lib().gbo_bmv_count_noalloc(b * 4, b * 4, b, limit + 1, None, None, None, None, None,
                                             gbo.OUT_I32, 0, None)
        assert st == ERR_UNSUPPORTED
        assert "scratch" in gbo.lib().gbo_last_error().decode()


@pytest.mark.parametrize("b", WIDTHS)
def test_noalloc_chunk_boundaries_hand_built(gbo, orc, gpu, b):
    """Block rows sized from the entry point's largest chunk, K = 32768 / b
    tiles (what large graphs run at): a row ending inside the first K tiles,
    a row crossing into the second, several short rows, an empty row, a row
    spanning at least three K, and short rows at the end.  A graph this small
    runs at the smallest chunk (64 tiles), so its long rows cross many chunk
    boundaries (slot 1 of their first chunk, slot 0 of the others) and short
    rows sit whole or split inside chunks.  Counts against the oracle, two
    calls in a row."""
    K = 32768 // b
    lens = [K // 2, K, 3, 5, 1, 0, 7, 3 * K + K // 3, 0, 2, 9]
    nbr = len(lens)
    nbc = 131072 // b  # room for 3K distinct ascending block columns
    rng = np.random.default_rng(900 + b)
    rowptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    colind = np.concatenate([np.sort(rng.choice(nbc, m, replace=False)) for m in lens]).astype(np.int32)
    top = (1 << b) - 1 if b < 64 else (1 << 64) - 1
    words = rng.integers(0, top, len(colind) * b, dtype=np.uint64, endpoint=True)
    words[rng.random(len(words)) < 0.3] = 0
    nrows, ncols = nbr * b, nbc * b
    ob = orc.B2SR(rowptr, colind, words, nrows, ncols, b)
    wd = ob.narrow()
    drp, dci, dv = (gbo.DeviceBuffer.from_numpy(a) for a in (rowptr, colind, wd))
    for call in range(2):
        x = (rng.random(ncols) < (0.5 if call == 0 else 0.15)).astype(np.int32)
        xw = orc.pack_vector(x, b)
        dx = gbo.DeviceBuffer.from_numpy(xw.astype(wd.dtype))
        y = gbo.DeviceBuffer.from_numpy(np.full(nrows, -3, np.int32))
        st = gbo.lib().gbo_bmv_count_noalloc(nrows, ncols, b, len(colind), drp.ptr, dci.ptr, dv.ptr, dx.ptr,
                                             y.ptr, gbo.OUT_I32, 0, None)
        gbo.check(st, "bmv_count_noalloc")
        assert np.array_equal(y.to_numpy(np.int32, nrows), orc.bmv_count(ob, xw)), (b, call)
