"""Failure paths, each made on the host (no GPU fault, trap or hang): an
injected host allocation failure, iteration loops stopped before the device
finishes, a wait that gives up, and admission past a bounded queue while the
server holds admission.  The reference has no failure handling at all (its
error checks compile away, algorithm/utility.cu:17-30)."""
import numpy as np
import pytest


def test_injected_host_allocation_failure_in_readers(gbo, tmp_path):
    p = tmp_path / "tri.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n3 3 3\n2 1\n3 1\n3 2\n")
    ok = gbo.read_mtx(str(p))
    assert ok.nnz == 6
    try:
        gbo.debug_inject(gbo.INJECT_HOST_ALLOC, 1)
        with pytest.raises(gbo.GboError) as e:
            gbo.read_mtx(str(p))
        assert e.value.status == gbo.GBO_ERR_NOMEM
        assert "allocation" in gbo.lib().gbo_last_error().decode()
        # armed for the second allocation: the first call succeeds, the next fails
        gbo.debug_inject(gbo.INJECT_HOST_ALLOC, 2)
        assert gbo.gen_rmat(8, 4, seed=1).nnz > 0
        with pytest.raises(gbo.GboError) as e:
            gbo.gen_er(100, 0.1, 1)
        assert e.value.status == gbo.GBO_ERR_NOMEM
    finally:
        gbo.debug_inject(gbo.INJECT_HOST_ALLOC, 0)
    # disarmed: the same calls work again and give the same result
    again = gbo.read_mtx(str(p))
    assert np.array_equal(again.rowptr, ok.rowptr) and np.array_equal(again.colind, ok.colind)


def test_injection_arguments(gbo):
    for what in (gbo.INJECT_HOST_ALLOC, gbo.INJECT_REPLAY_CAP, gbo.INJECT_SERVER_HOLD, gbo.INJECT_BARRIER_SKIP):
        assert gbo.lib().gbo_debug_inject(what, 1) == gbo.GBO_OK  # arming and disarming touch no GPU
        assert gbo.lib().gbo_debug_inject(what, 0) == gbo.GBO_OK
    assert gbo.lib().gbo_debug_inject(99, 1) == gbo.GBO_ERR_INVALID
    assert gbo.lib().gbo_debug_inject(gbo.INJECT_REPLAY_CAP, -1) == gbo.GBO_ERR_INVALID
    assert gbo.lib().gbo_status_string(gbo.GBO_ERR_FULL) == b"GBO_ERR_FULL"


@pytest.mark.gpu
def test_replay_cap_returns_timeout_then_recovers(gbo, orc, gpu):
    """A loop that is not finished after its replays returns GBO_ERR_TIMEOUT;
    the next call (cap lifted) starts afresh and is exact.  A path of 300
    vertices needs 300 BFS levels, far more than one replay of the captured
    levels holds."""
    m = 300
    path = gbo.csr_from_edges(np.arange(m - 1, dtype=np.int32), np.arange(1, m, dtype=np.int32), m, True, True)
    gp = gbo.Graph.from_csr(path, 32, gbo.FLAG_SYMMETRIC)
    csr = gbo.gen_rmat(12, 16, seed=3)
    g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_SYMMETRIC)
    calls = [lambda: gp.bfs(0), lambda: gp.msbfs(np.array([0] + [5] * 31, np.int32)),
             lambda: gp.sssp(0), lambda: g.pagerank(0.85, 40, -1.0)]
    try:
        gbo.debug_inject(gbo.INJECT_REPLAY_CAP, 1)
        for call in calls:
            with pytest.raises(gbo.GboError) as e:
                call()
            assert e.value.status == gbo.GBO_ERR_TIMEOUT
    finally:
        gbo.debug_inject(gbo.INJECT_REPLAY_CAP, 0)
    lv, depth = gp.bfs(0)
    assert depth == m and np.array_equal(lv, np.arange(m))
    ms = gp.msbfs(np.array([0] + [5] * 31, np.int32))
    ms = ms[0] if isinstance(ms, tuple) else ms
    assert np.array_equal(np.asarray(ms).reshape(m, 32)[:, 0], np.arange(m))
    lv, depth = g.bfs(0)
    assert np.array_equal(lv, orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, 0)[0])
    p, it = g.pagerank(0.85, 40, -1.0)
    outdeg = np.bincount(csr.colind, minlength=csr.nrows).astype(np.int32)
    ref, _ = orc.pagerank_f64(csr.rowptr, csr.colind, csr.nrows, outdeg, 0.85, 40, -1.0)
    assert it == 40 and np.abs(p - ref).sum() / np.abs(ref).sum() <= 1e-5


@pytest.mark.gpu
def test_cooperative_bfs_barrier_timeout_then_recovers(gbo, orc, gpu):
    """A block of the cooperative BFS that leaves before its first grid
    barrier: the other blocks' bounded wait (100 ms under the injection) runs
    out, they set the barrier error and return, and gbo_bfs reports
    GBO_ERR_TIMEOUT with the context usable.  The next BFS is exact."""
    csr = gbo.gen_rmat(14, 16, seed=4)
    g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_SYMMETRIC)
    g.set_bfs_loop(gbo.BFS_LOOP_COOP)
    ref = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, 0)[0]
    for skip in (1, 3):  # block 0 (which completes the arrival word) and block 2
        try:
            gbo.debug_inject(gbo.INJECT_BARRIER_SKIP, skip)
            with pytest.raises(gbo.GboError) as e:
                g.bfs(0)
            assert e.value.status == gbo.GBO_ERR_TIMEOUT
        finally:
            gbo.debug_inject(gbo.INJECT_BARRIER_SKIP, 0)
        lv, _ = g.bfs(0)
        assert np.array_equal(lv, ref)
        assert g.last_run()["kernel_launches"] == 2


@pytest.mark.gpu
def test_server_timeout_hold_and_bounded_queue(gbo, orc, gpu):
    """While admission is held, submissions queue up to the limit and the
    next one returns GBO_ERR_FULL; waits give up with GBO_ERR_TIMEOUT and
    polls answer GBO_ERR_NOTREADY; released, every queued query finishes
    with the exact result."""
    csr = gbo.gen_rmat(11, 16, seed=4)
    n = csr.nrows
    g = gbo.Graph.from_csr(csr, 32)
    srv = gbo.Server(g, bfs_slots=32, ppr_slots=0)
    try:
        gbo.debug_inject(gbo.INJECT_SERVER_HOLD, 1)
        srv.set_queue_limit(5)
        srcs = [0, 17, 99, 512, 2047]
        tickets = [srv.submit_bfs(s) for s in srcs]
        with pytest.raises(gbo.GboError) as e:
            srv.submit_bfs(3)
        assert e.value.status == gbo.GBO_ERR_FULL
        st = srv.stats()
        assert st["pending"] == 5 and st["in_flight"] == 0 and st["bfs_completed"] == 0
        with pytest.raises(gbo.GboError) as e:
            srv.wait(tickets[0], "bfs", timeout=0.05)
        assert e.value.status == gbo.GBO_ERR_TIMEOUT
        assert srv.poll(tickets[1], "bfs") is None  # GBO_ERR_NOTREADY
        # a ticket that was never issued only ever times out
        with pytest.raises(gbo.GboError) as e:
            srv.wait(10 ** 12, "bfs", timeout=0.02)
        assert e.value.status == gbo.GBO_ERR_TIMEOUT
    finally:
        gbo.debug_inject(gbo.INJECT_SERVER_HOLD, 0)
    for s, t in zip(srcs, tickets):
        lv, _, _ = srv.wait(t, "bfs", timeout=60.0)
        assert np.array_equal(lv, orc.bfs_csr(csr.rowptr, csr.colind, n, s)[0]), s
    srv.set_queue_limit(0)
    more = [srv.submit_bfs(int(s)) for s in range(40)]  # unbounded again
    for t in more:
        srv.wait(t, "bfs", timeout=60.0)
    assert srv.stats()["bfs_completed"] == 45
    srv.close()
