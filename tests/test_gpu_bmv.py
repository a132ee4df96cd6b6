"""BMV primitives on the GPU vs the oracle (bit-exact for integer semirings,
1e-5 relative for fp32), including block rows split across warps."""
import numpy as np
import pytest

from gpu_cases import cases

pytestmark = pytest.mark.gpu
WIDTHS = [4, 8, 16, 32, 64]
INF = 2147483647


@pytest.fixture(scope="module")
def graphs(gbo):
    return cases(gbo)


def _packed(gbo, orc, csr, b):
    return gbo.Graph.from_csr(csr, b), orc.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, b)


@pytest.mark.parametrize("b", WIDTHS)
def test_bmv_count(gbo, orc, gpu, graphs, b):
    rng = np.random.default_rng(b)
    for name, csr in graphs.items():
        g, ref = _packed(gbo, orc, csr, b)
        x = (rng.random(csr.ncols) < 0.5).astype(np.int32)
        xw = orc.pack_vector(x, b)
        y_ref = orc.bmv_count(ref, xw)
        dx = gbo.DeviceBuffer.from_numpy(xw.astype(gbo.WORD_DTYPE[b]))
        dy = gbo.DeviceBuffer(4 * csr.nrows)
        g.bmv_count(dx, dy)
        assert np.array_equal(dy.to_numpy(np.int32, csr.nrows), y_ref), (name, b)
        # accumulate (+=) into float output, like the reference's T=float C
        base = rng.integers(0, 5, csr.nrows).astype(np.float32)
        dyf = gbo.DeviceBuffer.from_numpy(base)
        g.bmv_count(dx, dyf, gbo.OUT_F32, accumulate=True)
        assert np.array_equal(dyf.to_numpy(np.float32, csr.nrows), base + y_ref), (name, b)


@pytest.mark.parametrize("b", WIDTHS)
def test_bmv_masked(gbo, orc, gpu, graphs, b):
    rng = np.random.default_rng(100 + b)
    for name, csr in graphs.items():
        g, ref = _packed(gbo, orc, csr, b)
        x = (rng.random(csr.ncols) < 0.05).astype(np.int32)
        m = (rng.random(csr.nrows) < 0.3).astype(np.int32)
        m[: min(3 * b, csr.nrows)] = 1  # fully masked block rows
        xw, mw = orc.pack_vector(x, b), orc.pack_vector(m, b)
        wd = gbo.WORD_DTYPE[b]
        dx = gbo.DeviceBuffer.from_numpy(xw.astype(wd))
        dm = gbo.DeviceBuffer.from_numpy(mw.astype(wd))
        do = gbo.DeviceBuffer(np.dtype(wd).itemsize * len(mw))
        for mask in (dm, None):
            g.bmv_masked(dx, mask, do)
            want = orc.bmv_masked(ref, xw, mw if mask is not None else None).astype(wd)
            assert np.array_equal(do.to_numpy(wd, len(mw)), want), (name, b, mask is None)


@pytest.mark.parametrize("b", WIDTHS)
def test_bmv_value_semirings(gbo, orc, gpu, graphs, b):
    rng = np.random.default_rng(200 + b)
    for name, csr in graphs.items():
        g, ref = _packed(gbo, orc, csr, b)
        n = csr.nrows
        # min-plus over uint32 with INF
        d = rng.integers(0, 50, n).astype(np.uint32)
        d[rng.random(n) < 0.4] = INF
        dd, dy = gbo.DeviceBuffer.from_numpy(d), gbo.DeviceBuffer(4 * n)
        g.bmv_minplus(dd, dy)
        assert np.array_equal(dy.to_numpy(np.uint32, n), orc.bmv_minplus(ref, d)), (name, b)
        # min-select over int32
        lab = rng.permutation(n).astype(np.int32)
        dl = gbo.DeviceBuffer.from_numpy(lab)
        g.bmv_minselect(dl, dy)
        assert np.array_equal(dy.to_numpy(np.int32, n), orc.bmv_minselect(ref, lab)), (name, b)
        # fp32: y = alpha * sum x*scale + add
        xf = rng.random(n).astype(np.float32)
        sc = (1.0 / np.maximum(1, np.bincount(csr.colind, minlength=n))).astype(np.float32)
        dxf, dsc = gbo.DeviceBuffer.from_numpy(xf), gbo.DeviceBuffer.from_numpy(sc)
        g.bmv_float(dxf, dy, 0.85, dsc, 0.01)
        got = dy.to_numpy(np.float32, n)
        # the oracle's fp32 restatement (reference term order) within 1e-5 on
        # rows of modest degree; every row within 1e-6 of the fp64 sum
        want = orc.bmv_float(ref, xf, 0.85, sc, 0.01)
        deg = np.diff(csr.rowptr)
        small = deg < 2000
        np.testing.assert_allclose(got[small], want[small], rtol=1e-5, atol=1e-7, err_msg=f"{name} b={b}")
        A = np.zeros((n, csr.ncols), np.float64)
        A[np.repeat(np.arange(n), deg), csr.colind] = 1
        want64 = 0.85 * (A @ (xf * sc).astype(np.float64)) + 0.01
        np.testing.assert_allclose(got, want64, rtol=1e-6, atol=1e-7, err_msg=f"{name} b={b}")
        # transposed fp32: y = alpha * P^T (x*scale) + add
        dyt = gbo.DeviceBuffer(4 * csr.ncols)
        g.bmv_float_transposed(dxf, dyt, 0.5, dsc, 0.25)
        want_t = 0.5 * (A.T @ (xf.astype(np.float64) * sc)) + 0.25
        np.testing.assert_allclose(dyt.to_numpy(np.float32, csr.ncols), want_t, rtol=1e-5, atol=1e-6)


def test_wrap_caller_owned_b2sr(gbo, orc, gpu, graphs):
    """gbo_graph_wrap_b2sr: reference-style caller-owned device B2SR."""
    csr = graphs["rmat14"]
    for b in WIDTHS:
        ref = orc.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, b)
        rp = gbo.DeviceBuffer.from_numpy(ref.rowptr)
        ci = gbo.DeviceBuffer.from_numpy(ref.colind)
        va = gbo.DeviceBuffer.from_numpy(ref.narrow())
        g = gbo.Graph.wrap_b2sr(csr.nrows, csr.ncols, b, 0, ref.nblk, rp, ci, va)
        x = (np.random.default_rng(1).random(csr.ncols) < 0.5).astype(np.int32)
        xw = orc.pack_vector(x, b)
        dx = gbo.DeviceBuffer.from_numpy(xw.astype(gbo.WORD_DTYPE[b]))
        dy = gbo.DeviceBuffer(4 * csr.nrows)
        g.bmv_count(dx, dy)
        assert np.array_equal(dy.to_numpy(np.int32, csr.nrows), orc.bmv_count(ref, xw))
        with pytest.raises(gbo.GboError):
            g.pagerank()  # wrapped without out-degrees
