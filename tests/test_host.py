"""CPU-side checks of libgbo: the C ABI loads and exports every symbol in
include/gbo.h, and the host input path (readers, CSR utilities, generators)
matches the oracle's restatements.  No device calls."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def header_symbols():
    with open(os.path.join(ROOT, "include", "gbo.h")) as f:
        src = f.read()
    return sorted(set(re.findall(r"GBO_API\s+[\w\s\*]*?\b(gbo_\w+)\s*\(", src)))


def test_library_exports_every_header_symbol(gbo):
    import ctypes

    lib = ctypes.CDLL(gbo.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 50
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # the Python binding declares every exported entry point
    assert set(syms) <= set(gbo.exported_symbols()), set(syms) - set(gbo.exported_symbols())


def test_status_strings(gbo):
    assert gbo.lib().gbo_status_string(0) == b"GBO_OK"
    assert gbo.lib().gbo_status_string(4) == b"GBO_ERR_UNSORTED"
    assert gbo.lib().gbo_version() >= 100


def test_mtx_errors(gbo, tmp_path):
    with pytest.raises(gbo.GboError) as e:
        gbo.read_mtx(str(tmp_path / "missing.mtx"))
    assert e.value.status == gbo.GBO_ERR_IO
    bad = tmp_path / "bad.mtx"
    bad.write_text("%%MatrixMarket matrix coordinate pattern general\n4 4 2\n1 2\n9 1\n")
    with pytest.raises(gbo.GboError) as e:
        gbo.read_mtx(str(bad))
    assert e.value.status == gbo.GBO_ERR_BOUNDS


@pytest.mark.parametrize("banner", ["pattern general", "pattern symmetric", "real symmetric",
                                    "integer general", "real hermitian"])
def test_mtx_readers_match_oracle(gbo, orc, tmp_path, banner):
    rng = np.random.default_rng(7)
    n = 70
    entries = [(int(rng.integers(1, n + 1)), int(rng.integers(1, n + 1))) for _ in range(400)]
    entries += [(3, 3), (5, 9), (5, 9)]  # a self-loop and a duplicate
    lines = [f"%%MatrixMarket matrix coordinate {banner}", "% comment", f"{n} {n} {len(entries)}"]
    val = "" if "pattern" in banner else " 1.5"
    lines += [f"{i} {j}{val}" for i, j in entries]
    p = tmp_path / "m.mtx"
    p.write_text("\n".join(lines) + "\n")
    for d in (0, 1, 2):
        nr, nc, rp, ci = orc.read_mtx_readmtx(str(p), d)
        c = gbo.read_mtx(str(p), gbo.MTX_READMTX, d)
        assert np.array_equal(c.rowptr, rp) and np.array_equal(c.colind, ci)
    nr, nc, rp, ci = orc.read_mtx_mmio(str(p))
    c = gbo.read_mtx(str(p), gbo.MTX_MMIO, 0)
    assert np.array_equal(c.rowptr, rp) and np.array_equal(c.colind, ci)


def test_readmtx_respects_selfloop_env(gbo, orc, tmp_path, monkeypatch):
    p = tmp_path / "s.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern general\n3 3 3\n1 1\n1 2\n2 3\n")
    monkeypatch.setenv("GRB_UTIL_REMOVE_SELFLOOP", "0")
    c = gbo.read_mtx(str(p), gbo.MTX_READMTX, 0)
    nr, nc, rp, ci = orc.read_mtx_readmtx(str(p), 0, remove_self_loops=False)
    assert c.nnz == 3 and np.array_equal(c.colind, ci)


def test_generators_are_simple_symmetric_and_seeded(gbo):
    for csr in (gbo.gen_rmat(10, 16, seed=1), gbo.gen_er(500, 0.02, 3), gbo.gen_er_avgdeg(700, 8, 4),
                gbo.gen_king_mesh(9)):
        n = csr.nrows
        rows = np.repeat(np.arange(n), np.diff(csr.rowptr))
        assert np.all(rows != csr.colind), "self-loop"
        for r in range(n):
            seg = csr.colind[csr.rowptr[r]:csr.rowptr[r + 1]]
            assert np.all(np.diff(seg) > 0), "row not strictly ascending"
        a = set(zip(rows.tolist(), csr.colind.tolist()))
        assert all((j, i) in a for i, j in a), "not symmetric"
    a1, a2 = gbo.gen_rmat(11, 16, seed=9), gbo.gen_rmat(11, 16, seed=9)
    assert np.array_equal(a1.colind, a2.colind)
    assert not np.array_equal(a1.colind, gbo.gen_rmat(11, 16, seed=10).colind)


def test_rmat_generator_matches_python_restatement(gbo):
    """Bit-exact check of the R-MAT stream definition at a small scale."""
    M64 = (1 << 64) - 1

    def splitmix(s):
        s = (s + 0x9E3779B97F4A7C15) & M64
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return s, z ^ (z >> 31)

    def rotl(x, k):
        return ((x << k) | (x >> (64 - k))) & M64

    def stream(seed, k):
        sm = seed ^ ((k * 0xD1B54A32D192ED03) & M64)
        st = []
        for _ in range(4):
            sm, z = splitmix(sm)
            st.append(z)
        return st

    def nxt(s):
        res = (rotl((s[1] * 5) & M64, 7) * 9) & M64
        t = (s[1] << 17) & M64
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45)
        return res

    scale, ef, seed = 6, 4, 11
    a, b, c = 0.57, 0.19, 0.19
    src, dst = [], []
    for k in range((1 << scale) * ef):
        s = stream(seed, k)
        u = v = 0
        for _ in range(scale):
            r = (nxt(s) >> 11) * 2.0 ** -53
            u = (u << 1) | (r >= a + b)
            v = (v << 1) | ((a <= r < a + b) or r >= a + b + c)
        src.append(u)
        dst.append(v)
    ref = gbo.csr_from_edges(src, dst, 1 << scale, True, True)
    got = gbo.gen_rmat(scale, ef, a, b, c, seed)
    assert np.array_equal(ref.rowptr, got.rowptr) and np.array_equal(ref.colind, got.colind)


@pytest.mark.parametrize("scale,ef,seed,abc", [(6, 4, 11, (0.57, 0.19, 0.19)),
                                               (12, 16, 0, (0.57, 0.19, 0.19)),
                                               (15, 16, 2, (0.57, 0.19, 0.19)),
                                               (13, 8, 5, (0.45, 0.15, 0.15))])
def test_oracle_rmat_generator_equals_library(gbo, orc, scale, ef, seed, abc):
    """The CPU legs of the benchmark build their R-MAT inputs with the
    oracle's generator (no product library); it must give the library's
    graph array for array."""
    a, b, c = abc
    got = orc.gen_rmat(scale, ef, a, b, c, seed)
    ref = gbo.gen_rmat(scale, ef, a, b, c, seed)
    assert got.nrows == ref.nrows and got.nnz == ref.nnz
    assert np.array_equal(got.rowptr, ref.rowptr) and np.array_equal(got.colind, ref.colind)


def test_csr_transpose_and_tril(gbo):
    rng = np.random.default_rng(2)
    src = rng.integers(0, 50, 300)
    dst = rng.integers(0, 50, 300)
    csr = gbo.csr_from_edges(src, dst, 50, symmetrize=False, drop_self_loops=False)
    t = csr.transpose()
    dense = np.zeros((50, 50), np.int32)
    dense[np.repeat(np.arange(50), np.diff(csr.rowptr)), csr.colind] = 1
    dt = np.zeros((50, 50), np.int32)
    dt[np.repeat(np.arange(50), np.diff(t.rowptr)), t.colind] = 1
    assert np.array_equal(dense.T, dt)
    low = csr.tril()
    dl = np.zeros((50, 50), np.int32)
    dl[np.repeat(np.arange(50), np.diff(low.rowptr)), low.colind] = 1
    assert np.array_equal(np.tril(dense), dl)


def test_mesh_edge_count_closed_form(gbo):
    m = gbo.gen_king_mesh(64)
    assert m.nnz // 2 == 2 * 64 * 63 + 2 * 63 * 63


def test_null_handles_are_rejected_without_a_gpu(gbo):
    """The setters validate their arguments on the host: a NULL graph or
    server handle is GBO_ERR_INVALID, with no device touched."""
    lib = gbo.lib()
    assert lib.gbo_graph_set_bfs_loop(None, gbo.BFS_LOOP_COOP, 0) == gbo.GBO_ERR_INVALID
    assert lib.gbo_graph_set_bfs_direction(None, 1, -1) == gbo.GBO_ERR_INVALID
    assert lib.gbo_server_set_admission(None, ctypes.c_float(0.5)) == gbo.GBO_ERR_INVALID
    assert lib.gbo_server_set_queue_limit(None, 10) == gbo.GBO_ERR_INVALID
