"""The reference's own kernels (compiled for sm_100a from the reference
sources into oracle/_ref by oracle/Makefile) run on B2SR packed by libgbo and
compared with libgbo's kernels.  This pins the packed layout and the BMV /
masked-BMM semantics to the reference's code, not only to the restatement.
Graphs stay small: the reference kernels use int32 word offsets."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT
from gpu_cases import cases

pytestmark = pytest.mark.gpu
REF = os.path.join(ROOT, "oracle", "_ref")
INF = 2147483647


def _load(name):
    p = os.path.join(REF, name)
    if not os.path.exists(p):
        pytest.skip(f"{p} not built (needs the reference checkout at build time)")
    return C.CDLL(p)


@pytest.fixture(scope="module")
def refbmv(gpu):
    return _load("librefbmv.so")


@pytest.fixture(scope="module")
def refbmm(gpu):
    return _load("librefbmm.so")


@pytest.fixture(scope="module")
def graphs(gbo):
    cs = cases(gbo)
    cs.pop("single")
    return cs


def _dev_b2sr(gbo, g):
    r, c, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
    gbo.check(gbo.lib().gbo_graph_b2sr(g.h, C.byref(r), C.byref(c), C.byref(v)))
    return r.value, c.value, v.value


def _pad(a, n, fill):
    out = np.full(n, fill, dtype=a.dtype)
    out[: len(a)] = a
    return out


@pytest.mark.parametrize("b,fn", [(4, "ref_bmv4_sparse"), (8, "ref_bmv8_sparse"),
                                  (16, "ref_bmv16_sparse_new"), (32, "ref_bmv32_sparse_new"),
                                  (64, "ref_bmv64_sparse_new")])
def test_reference_count_kernels_on_our_packing(gbo, refbmv, graphs, b, fn):
    rng = np.random.default_rng(b)
    for name, csr in graphs.items():
        g = gbo.Graph.from_csr(csr, b)
        inf = g.info()
        r, c, v = _dev_b2sr(gbo, g)
        x = (rng.random(csr.ncols) < 0.5).astype(np.int32)
        xw = gbo.bits_from_numpy(x, b)
        dx = gbo.DeviceBuffer.from_numpy(_pad(xw, inf.nblockcols + 64, 0))
        npad = (inf.nblockrows + 64) * b
        dref = gbo.DeviceBuffer.zeros(4 * npad)
        f = getattr(refbmv, fn)
        f.argtypes = [C.c_void_p] * 5 + [C.c_int, C.c_int]
        assert f(v, dx.ptr, dref.ptr, r, c, inf.nblockrows, int(inf.nblocks)) == 0
        assert refbmv.ref_sync() == 0
        got_ref = dref.to_numpy(np.float32, csr.nrows).astype(np.int64)
        dy = gbo.DeviceBuffer(4 * csr.nrows)
        g.bmv_count(dx, dy)
        assert np.array_equal(dy.to_numpy(np.int32, csr.nrows), got_ref), (name, b)


def test_reference_masked_v4_on_our_packing(gbo, refbmv, graphs):
    rng = np.random.default_rng(7)
    f = refbmv.ref_bmv32_sparse_bin_masked_v4
    f.argtypes = [C.c_void_p] * 5 + [C.c_int, C.c_void_p]
    for name, csr in graphs.items():
        g = gbo.Graph.from_csr(csr, 32)
        inf = g.info()
        r, c, v = _dev_b2sr(gbo, g)
        x = (rng.random(csr.ncols) < 0.1).astype(np.int32)
        m = (rng.random(csr.nrows) < 0.3).astype(np.int32)
        dx = gbo.DeviceBuffer.from_numpy(gbo.bits_from_numpy(x, 32))
        dm = gbo.DeviceBuffer.from_numpy(gbo.bits_from_numpy(m, 32))
        dref = gbo.DeviceBuffer.zeros(4 * inf.nblockrows)  # rows without tiles stay 0
        assert f(v, dx.ptr, dref.ptr, r, c, inf.nblockrows, dm.ptr) == 0
        assert refbmv.ref_sync() == 0
        dout = gbo.DeviceBuffer(4 * inf.nblockrows)
        g.bmv_masked(dx, dm, dout)
        assert np.array_equal(dout.to_numpy(np.uint32), dref.to_numpy(np.uint32)), name


def test_reference_minplus_and_float_on_our_packing(gbo, refbmv, graphs):
    rng = np.random.default_rng(8)
    fmp = refbmv.ref_bmv32_sparse_full_minplus
    fmp.argtypes = [C.c_void_p] * 5 + [C.c_int]
    ffl = refbmv.ref_bmv32_sparse_full
    ffl.argtypes = [C.c_void_p] * 5 + [C.c_int, C.c_void_p, C.c_float]
    for name, csr in graphs.items():
        g = gbo.Graph.from_csr(csr, 32)
        inf = g.info()
        r, c, v = _dev_b2sr(gbo, g)
        npad = inf.nblockrows * 32
        n = csr.nrows
        # min-plus: compare rows whose block row stores its diagonal tile (the
        # reference adds the 0-weight diagonal only there)
        d = rng.integers(0, 40, n).astype(np.uint32)
        d[rng.random(n) < 0.3] = INF
        dd = gbo.DeviceBuffer.from_numpy(_pad(d, npad, np.uint32(INF)))
        dref = gbo.DeviceBuffer.from_numpy(np.full(npad, 77, np.uint32))
        assert fmp(v, dd.ptr, dref.ptr, r, c, inf.nblockrows) == 0
        assert refbmv.ref_sync() == 0
        dy = gbo.DeviceBuffer(4 * n)
        g.bmv_minplus(gbo.DeviceBuffer.from_numpy(d), dy)
        rp, ci, _ = g.b2sr()
        diag = np.array([R in ci[rp[R]:rp[R + 1]] for R in range(inf.nblockrows)])
        rows = np.repeat(diag, 32)[:n]
        ours = dy.to_numpy(np.uint32, n)
        assert np.array_equal(ours[rows], dref.to_numpy(np.uint32, n)[rows]), name
        # fp32 PageRank BMV as pr.cu uses it: P = A^T (CSC packing) and the
        # degree of column j read from A's CSR row pointer
        gt = gbo.Graph.from_csr(csr, 32, gbo.FLAG_TRANSPOSE)
        tr, tc, tv = _dev_b2sr(gbo, gt)
        p = rng.random(n).astype(np.float32)
        dp = gbo.DeviceBuffer.from_numpy(_pad(p, npad, np.float32(0)))
        rpp = _pad(csr.rowptr, npad + 1, csr.rowptr[-1])  # reads every column of a tile
        drp = gbo.DeviceBuffer.from_numpy(rpp)
        dref = gbo.DeviceBuffer.zeros(4 * npad)
        assert ffl(tv, dp.ptr, dref.ptr, tr, tc, inf.nblockrows, drp.ptr, 0.85) == 0
        assert refbmv.ref_sync() == 0
        dy = gbo.DeviceBuffer(4 * n)
        gbo.check(gbo.lib().gbo_bmv_float_degptr(gt.h, dp.ptr, dy.ptr, 0.85, drp.ptr, None))
        np.testing.assert_allclose(dy.to_numpy(np.float32, n), dref.to_numpy(np.float32, n),
                                   rtol=2e-5, atol=1e-7, err_msg=name)


def test_reference_masked_bmm_triangles_on_our_packing(gbo, refbmm, graphs):
    f = refbmm.ref_bmm32_sparse_masked_v5
    f.argtypes = [C.c_void_p] * 7 + [C.c_int, C.c_int, C.c_int]
    for name in ("er1000", "rmat12", "mesh33", "star20000"):
        csr = graphs[name]
        low = csr.tril()
        gl = gbo.Graph.from_csr(low, 32)                              # A: L, ROW layout
        glt = gbo.Graph.from_csr(low.transpose(), 32, gbo.FLAG_LAYOUT_COL)  # B: L^T, COL layout
        ar, ac, av = _dev_b2sr(gbo, gl)
        br, bc, bv = _dev_b2sr(gbo, glt)
        inf = gl.info()
        dcount = gbo.DeviceBuffer.zeros(4)
        assert f(av, bv, dcount.ptr, ar, ac, br, bc, inf.nblockrows, int(inf.nblocks), csr.nrows) == 0
        assert refbmm.ref_bmm_sync() == 0
        ref_tri = int(dcount.to_numpy(np.int32, 1)[0])
        ours = gbo.Graph.from_csr(csr, 32, gbo.FLAG_LOWER).tc()
        assert ours == ref_tri, name
