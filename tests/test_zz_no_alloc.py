"""gbo_bmv_count_noalloc (static device scratch, no allocation) against
gbo_bmv_count on the same packed graphs: identical integer counts, two calls
in a row with different vectors so that stale scratch would show.  The file
is named to be collected last; it also passes alone in a fresh process."""
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
def test_noalloc_matches_bmv_count(gbo, gpu, b):
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
            assert np.array_equal(y.to_numpy(np.int32, n), ref), (b, n, call)
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
