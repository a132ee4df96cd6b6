"""Matrix Market ingestion on the GPU (gbo_read_mtx_device / gbo_graph_from_mtx)
gives the host reader's CSR -- readMtx and mmio_data semantics, every
`directed` mode -- on generated files with comments, blank lines, CRLF line
ends, values, duplicates and self-loops, and the host reader's error codes on
malformed files."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _write(path, banner, n, m, pairs, rng, crlf=False, values=False, blanks=False):
    nl = "\r\n" if crlf else "\n"
    lines = [banner, "% generated", "%"]
    lines.append(f"{n} {m} {len(pairs)}")
    for i, j in pairs:
        s = f"{i + 1} {j + 1}"
        if values:
            s += f" {rng.random():.6f}"
        if rng.random() < 0.1:
            s = "  \t" + s + "  "
        lines.append(s)
        if blanks and rng.random() < 0.05:
            lines.append("   ")
    path.write_text(nl.join(lines) + nl)


def _pairs(rng, n, m, count, self_loops=True, dups=True):
    i = rng.integers(0, n, count)
    j = rng.integers(0, m, count)
    if self_loops:
        k = rng.choice(count, count // 20, replace=False)
        j[k] = np.minimum(i[k], m - 1)
    p = list(zip(i.tolist(), j.tolist()))
    if dups:
        p += p[: count // 10]
    return p


def _same(a, b):
    return (a.nrows == b.nrows and a.ncols == b.ncols and np.array_equal(a.rowptr, b.rowptr)
            and np.array_equal(a.colind, b.colind))


@pytest.mark.parametrize("crlf", [False, True])
def test_gpu_reader_matches_host_reader(gbo, gpu, tmp_path, crlf):
    rng = np.random.default_rng(1 if crlf else 2)
    cases = [
        ("%%MatrixMarket matrix coordinate pattern symmetric", 500, 500, _pairs(rng, 500, 500, 4000)),
        ("%%MatrixMarket matrix coordinate real general", 700, 300, _pairs(rng, 700, 300, 5000)),
        ("%%MatrixMarket matrix coordinate integer symmetric", 64, 64, _pairs(rng, 64, 64, 200)),
        ("%%MatrixMarket matrix coordinate pattern general", 10, 10, []),
    ]
    for k, (banner, n, m, pairs) in enumerate(cases):
        path = tmp_path / f"m{k}.mtx"
        _write(path, banner, n, m, pairs, rng, crlf=crlf, values="real" in banner or "integer" in banner,
               blanks=True)
        for mode in (gbo.MTX_READMTX, gbo.MTX_MMIO):
            for directed in ((0, 1, 2) if mode == gbo.MTX_READMTX else (0,)):
                host = gbo.read_mtx(str(path), mode, directed)
                dev = gbo.read_mtx_device(str(path), mode, directed)
                assert _same(host, dev), (banner, mode, directed)


def test_graph_from_mtx_is_graph_from_host_csr(gbo, gpu, tmp_path):
    csr = gbo.gen_rmat(12, 8, seed=5)
    rows = np.repeat(np.arange(csr.nrows), np.diff(csr.rowptr))
    keep = rows >= csr.colind  # one triangle, the banner says symmetric
    path = tmp_path / "rmat12.mtx"
    rng = np.random.default_rng(3)
    _write(path, "%%MatrixMarket matrix coordinate pattern symmetric", csr.nrows, csr.ncols,
           list(zip(rows[keep].tolist(), csr.colind[keep].tolist())), rng)
    g_dev = gbo.Graph.from_mtx(str(path), gbo.MTX_READMTX, 0, 32, gbo.FLAG_SYMMETRIC)
    g_host = gbo.Graph.from_csr(gbo.read_mtx(str(path)), 32, gbo.FLAG_SYMMETRIC)
    for a0, a1 in zip(g_dev.b2sr(), g_host.b2sr()):
        assert np.array_equal(a0, a1)
    assert np.array_equal(g_dev.bfs(0)[0], g_host.bfs(0)[0])
    g_dev.free()
    g_host.free()


def test_gpu_reader_errors_match_host(gbo, gpu, tmp_path):
    bad = {
        "short": "%%MatrixMarket matrix coordinate pattern general\n3 3 4\n1 2\n2 3\n",
        "bounds": "%%MatrixMarket matrix coordinate pattern general\n3 3 2\n1 2\n4 1\n",
        "malformed": "%%MatrixMarket matrix coordinate pattern general\n3 3 2\n1 2\nx y\n",
        "banner": "%%NotMatrixMarket\n3 3 1\n1 1\n",
    }
    for name, text in bad.items():
        p = tmp_path / f"{name}.mtx"
        p.write_text(text)
        with pytest.raises(gbo.GboError) as eh:
            gbo.read_mtx(str(p))
        with pytest.raises(gbo.GboError) as ed:
            gbo.read_mtx_device(str(p))
        assert eh.value.status == ed.value.status, name
