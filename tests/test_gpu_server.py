"""Continuous-batching query server: results vs the oracle, and each result
identical alone and in the mix of concurrently running queries."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l1(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).sum() / np.abs(b).sum())


def make_queries(n, nb, np_, seed):
    rng = np.random.default_rng(seed)
    qs = []
    for _ in range(nb):
        qs.append(("bfs", int(rng.integers(0, n))))
    for _ in range(np_):
        m = int(rng.integers(1, 65))
        verts = rng.choice(n, m, replace=False).astype(np.int32)
        wts = rng.dirichlet(np.ones(m)).astype(np.float32)
        qs.append(("ppr", (verts, wts)))
    order = rng.permutation(len(qs))
    return [qs[i] for i in order]


def submit_all(srv, qs, threads=2):
    tickets = [None] * len(qs)

    def run(part):
        for i in part:
            kind, arg = qs[i]
            tickets[i] = srv.submit_bfs(arg) if kind == "bfs" else srv.submit_ppr(*arg)

    parts = [range(t, len(qs), threads) for t in range(threads)]
    ths = [threading.Thread(target=run, args=(p,)) for p in parts]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    return tickets


def test_server_results_match_oracle_and_are_mix_independent(gbo, orc, gpu):
    csr = gbo.gen_rmat(12, 16, seed=0)
    n = csr.nrows
    outdeg = np.bincount(csr.colind, minlength=n).astype(np.int32)
    g = gbo.Graph.from_csr(csr, 32)
    qs = make_queries(n, 150, 40, seed=11)
    srv = gbo.Server(g, bfs_slots=64, ppr_slots=32, alpha=0.85, tol=1e-7)
    tickets = submit_all(srv, qs)
    mixed = []
    for (kind, arg), t in zip(qs, tickets):
        res, lat, it = srv.wait(t, kind)
        assert lat >= 0 and it >= 1
        mixed.append(res)
    st = srv.stats()
    assert st["bfs_completed"] == 150 and st["ppr_completed"] == 40 and st["in_flight"] == 0
    srv.close()
    for (kind, arg), res in zip(qs, mixed):
        if kind == "bfs":
            want, _ = orc.bfs_csr(csr.rowptr, csr.colind, n, arg)
            assert np.array_equal(res, want), arg
        else:
            v = np.zeros(n)
            v[arg[0]] = arg[1]
            want, _ = orc.ppr_f64(csr.rowptr, csr.colind, n, outdeg, v, 0.85, 1e-13)
            assert rel_l1(res, want) <= 1e-5
    # each query alone on a fresh server gives the same bits as in the mix
    srv1 = gbo.Server(g, bfs_slots=64, ppr_slots=32, alpha=0.85, tol=1e-7)
    for idx in [i for i, q in enumerate(qs) if q[0] == "ppr"][:5] + [i for i, q in enumerate(qs) if q[0] == "bfs"][:5]:
        kind, arg = qs[idx]
        t = srv1.submit_bfs(arg) if kind == "bfs" else srv1.submit_ppr(*arg)
        alone, _, _ = srv1.wait(t, kind)
        assert np.array_equal(alone, mixed[idx]), (kind, idx)
    srv1.close()


def test_server_poll_and_errors(gbo, gpu):
    g = gbo.Graph.from_csr(gbo.gen_er(1000, 0.02002, 0), 32)
    srv = gbo.Server(g, bfs_slots=32, ppr_slots=0)
    t = srv.submit_bfs(0)
    got = None
    for _ in range(100000):
        got = srv.poll(t, "bfs")
        if got is not None:
            break
    assert got is not None and got[0][0] == 0
    with pytest.raises(gbo.GboError):
        srv.submit_ppr([1], [1.0])  # no PPR slots
    with pytest.raises(gbo.GboError):
        srv.submit_bfs(10**6)
    srv.close()


def test_server_results_collected_in_any_order(gbo, orc, gpu):
    """More finished queries than pinned result buffers, collected newest
    first: results left uncollected move to heap memory instead of blocking
    retirement, and every result is still exact."""
    csr = gbo.gen_er(3000, 0.003, 5)
    g = gbo.Graph.from_csr(csr, 32)
    srv = gbo.Server(g, bfs_slots=64, ppr_slots=0)
    srcs = np.random.default_rng(12).integers(0, csr.nrows, 400)
    tickets = [srv.submit_bfs(int(s)) for s in srcs]
    out = {}
    for s, t in reversed(list(zip(srcs, tickets))):
        out[t] = (s, srv.wait(t, "bfs", timeout=60.0)[0])
    assert srv.stats()["bfs_completed"] == 400
    srv.close()
    for s, lv in out.values():
        assert np.array_equal(lv, orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, int(s))[0])


def test_server_device_delivery_matches_host_delivery(gbo, orc, gpu):
    """gbo_server_wait_device writes the same result into a device buffer as
    gbo_server_wait writes into host memory (BFS byte levels widened on the
    GPU, PPR values copied)."""
    csr = gbo.gen_rmat(12, 16, seed=1)
    n = csr.nrows
    g = gbo.Graph.from_csr(csr, 32)
    qs = make_queries(n, 60, 12, seed=12)
    srv = gbo.Server(g, bfs_slots=64, ppr_slots=32, alpha=0.85, tol=1e-7)
    t_host = submit_all(srv, qs)
    t_dev = submit_all(srv, qs)
    dbuf = gbo.DeviceBuffer(4 * n)
    for (kind, arg), th, td in zip(qs, t_host, t_dev):
        host, _, _ = srv.wait(th, kind)
        lat, it = srv.wait_device(td, dbuf)
        assert lat >= 0 and it >= 1
        dev = gbo.device_to_numpy(dbuf.ptr, np.int32 if kind == "bfs" else np.float32, n)
        assert np.array_equal(dev, host), (kind, arg if kind == "bfs" else len(arg[0]))
        if kind == "bfs":
            want, _ = orc.bfs_csr(csr.rowptr, csr.colind, n, arg)
            assert np.array_equal(dev, want)
    srv.close()


def test_server_byte_levels_match_int32_levels(gbo, orc, gpu):
    """gbo_server_wait_u8 delivers the same levels as bytes (255 =
    unreachable), into numpy memory and into pinned memory; a query deeper
    than 254 levels is refused with GBO_ERR_OVERFLOW and stays collectable
    as int32; a PPR ticket is refused."""
    import ctypes as C

    csr = gbo.gen_rmat(12, 16, seed=7)
    n = csr.nrows
    g = gbo.Graph.from_csr(csr, 32)
    srv = gbo.Server(g, bfs_slots=64, ppr_slots=32)
    srcs = np.random.default_rng(21).integers(0, n, 40)
    t8 = [srv.submit_bfs(int(s)) for s in srcs]
    t32 = [srv.submit_bfs(int(s)) for s in srcs]
    pin = C.c_void_p()
    gbo.check(gbo.lib().gbo_host_alloc(C.byref(pin), n), "host_alloc")
    try:
        for i, (s, a, b) in enumerate(zip(srcs, t8, t32)):
            if i % 2:
                got, lat, it = srv.wait_u8(a, out=pin.value)
                got = np.ctypeslib.as_array(C.cast(pin.value, C.POINTER(C.c_uint8)), (n,)).copy()
            else:
                got, lat, it = srv.wait_u8(a)
            want, _, _ = srv.wait(b, "bfs")
            assert np.array_equal(np.where(got == 255, -1, got.astype(np.int32)), want), int(s)
            assert np.array_equal(want, orc.bfs_csr(csr.rowptr, csr.colind, n, int(s))[0])
        tp = srv.submit_ppr([1, 2], [0.5, 0.5])
        with pytest.raises(gbo.GboError) as e:
            srv.wait_u8(tp)
        assert e.value.status == gbo.GBO_ERR_INVALID
        srv.wait(tp, "ppr")
    finally:
        gbo.lib().gbo_host_free(pin.value)
    srv.close()
    m = 300  # a path: 299 levels
    path = gbo.csr_from_edges(np.arange(m - 1, dtype=np.int32), np.arange(1, m, dtype=np.int32), m, True, True)
    gp = gbo.Graph.from_csr(path, 32)
    sp = gbo.Server(gp, bfs_slots=32, ppr_slots=0)
    t = sp.submit_bfs(0)
    with pytest.raises(gbo.GboError) as e:
        sp.wait_u8(t)
    assert e.value.status == gbo.GBO_ERR_OVERFLOW
    lv, _, _ = sp.wait(t, "bfs")
    assert np.array_equal(lv, np.arange(m))
    sp.close()


@pytest.mark.parametrize("admit", [0.0, 0.5, 1.0])
def test_server_admission_batching_keeps_results(gbo, orc, gpu, admit):
    """Admission into any free slot, into half-free engines or only into idle
    ones: every BFS result is the oracle's levels."""
    csr = gbo.gen_rmat(12, 16, seed=3)
    n = csr.nrows
    g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_SYMMETRIC)
    srv = gbo.Server(g, bfs_slots=64, ppr_slots=0)
    srv.set_admission(admit)
    srcs = np.random.default_rng(7).integers(0, n, 200)
    tickets = [srv.submit_bfs(int(s)) for s in srcs]
    for s, t in zip(srcs, tickets):
        res, _, _ = srv.wait(t, "bfs")
        assert np.array_equal(res, orc.bfs_csr(csr.rowptr, csr.colind, n, int(s))[0]), (admit, int(s))
    with pytest.raises(gbo.GboError):
        srv.set_admission(1.5)
    srv.close()
    g.free()


@pytest.mark.gpu
def test_server_batch_mode_switches_and_deep_queries(gbo, orc, gpu):
    """Batch mode (admission 1: each batch one multi-source BFS) with 256
    slots, switched to round-by-round admission and back while queries are
    in flight: every result is the oracle's levels, isolated sources
    included.  On a path of 300 vertices a batch query deeper than 254
    levels lands in the word pool (wait_u8 answers GBO_ERR_OVERFLOW)."""
    csr = gbo.gen_rmat(12, 16, seed=5)
    n = csr.nrows
    g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_SYMMETRIC)
    srv = gbo.Server(g, bfs_slots=256, ppr_slots=0)
    rng = np.random.default_rng(21)
    deg = np.diff(csr.rowptr)
    iso = np.flatnonzero(deg == 0)[:4]
    srcs, tickets = [], []
    for admit in (1.0, 0.0, 1.0, 0.5, 1.0):
        srv.set_admission(admit)
        part = rng.integers(0, n, 300)
        if admit == 1.0 and len(iso):
            part[: len(iso)] = iso
        srcs += [int(x) for x in part]
        tickets += [srv.submit_bfs(int(x)) for x in part]
    for s, t in zip(srcs, tickets):
        res, _, _ = srv.wait(t, "bfs")
        assert np.array_equal(res, orc.bfs_csr(csr.rowptr, csr.colind, n, s)[0]), s
    st = srv.stats()
    assert st["bfs_completed"] == len(srcs)
    srv.close()
    g.free()
    m = 300
    path = gbo.csr_from_edges(np.arange(m - 1, dtype=np.int32), np.arange(1, m, dtype=np.int32), m, True, True)
    gp = gbo.Graph.from_csr(path, 32, gbo.FLAG_SYMMETRIC)
    sp = gbo.Server(gp, bfs_slots=64, ppr_slots=0)
    sp.set_admission(1.0)
    t0, t1 = sp.submit_bfs(0), sp.submit_bfs(150)
    with pytest.raises(gbo.GboError) as e:
        sp.wait_u8(t0)
    assert e.value.status == gbo.GBO_ERR_OVERFLOW
    lv, _, _ = sp.wait(t0, "bfs")
    assert np.array_equal(lv, np.arange(m))
    lv, _, _ = sp.wait(t1, "bfs")
    assert np.array_equal(lv, np.abs(np.arange(m) - 150))
    sp.close()
    gp.free()
