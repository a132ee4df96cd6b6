"""Multi-process paths on the CPU (gloo, world size 2): the benchmark runs
one replica per GPU with no data-path collective; its ranks meet only at the
host barrier and the max-over-ranks reduction of the timed region, and the
reference arm runs on rank 0 alone.  The block-row sharded BFS exchanges
frontier words and counts between ranks (the library's gbo_bfs_shard_loop,
here over gloo with the oracle's level step)."""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2")
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist(2)
    d.barrier()
    got = d.max(10.0 + rank)  # per-rank timed-region ms; the job time is the max
    d.barrier()
    d.close()
    q.put((rank, got))


def test_dist_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=180)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: 11.0, 1: 11.0}


def test_reference_arm_rank0_only_under_torchrun():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--scale", "10", "--steps", "1", "--warmup", "3"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["e2e"]["h2d_bytes_per_step"] == 0 and rec["cpu_baseline"]["kind"] in ("port", "reference")


def _shard_rank(rank, port, q, b):
    """One gloo rank: the library's sharded-BFS loop (gbo_bfs_shard_loop)
    driven by the oracle's CPU twin of the level step, counts summed and
    next-frontier words all-gathered over gloo."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2")
    sys.path.insert(0, os.path.join(ROOT, "graph-bit-ops_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ctypes as C

    import numpy as np
    import torch
    import torch.distributed as dist

    import gbo
    import oracle
    import shard

    dist.init_process_group("gloo")
    csr = gbo.gen_rmat(10, 8, seed=4)
    n = csr.nrows
    bounds = shard.partition_rows(csr.rowptr, n, 2, b)
    r0, r1 = bounds[rank], bounds[rank + 1]
    part = shard.shard_csr(csr, r0, r1)
    nbr_all = (n + b - 1) // b
    wbound = [x // b if x < n else nbr_all for x in bounds]
    width = max(1, max(wbound[s + 1] - wbound[s] for s in range(2)))
    front = np.zeros(nbr_all, np.uint64)
    visited = np.zeros(max(1, wbound[rank + 1] - wbound[rank]), np.uint64)
    nxt = np.zeros_like(visited)
    level = np.full(max(1, r1 - r0), -1, np.int32)
    src = 5
    front[src // b] = np.uint64(1) << np.uint64(b - 1 - src % b)
    if r0 <= src < r1:
        visited[src // b - r0 // b] = front[src // b]
        level[src - r0] = 0

    def level_fn(user, lvl, count):
        count[0] = oracle.bfs_shard_level(part.rowptr, part.colind, r1 - r0, b, front, visited, level, lvl, nxt)
        return 0

    def allreduce_fn(user, value):
        t = torch.tensor([value[0]], dtype=torch.float64)  # exact below 2^53
        dist.all_reduce(t)
        value[0] = int(t.item())
        return 0

    def exchange_fn(user):
        mine = torch.zeros(width, dtype=torch.int64)
        k = wbound[rank + 1] - wbound[rank]
        mine[:k] = torch.from_numpy(nxt[:k].view(np.int64))
        parts = [torch.zeros(width, dtype=torch.int64) for _ in range(2)]
        dist.all_gather(parts, mine)
        for s_ in range(2):
            lo, hi = wbound[s_], wbound[s_ + 1]
            front[lo:hi] = parts[s_].numpy()[:hi - lo].view(np.uint64)
        return 0

    ops = gbo.ShardOps(None, gbo.SHARD_LEVEL_FN(level_fn), gbo.SHARD_ALLREDUCE_FN(allreduce_fn),
                       gbo.SHARD_EXCHANGE_FN(exchange_fn))
    depth = C.c_int(0)
    st = gbo.lib().gbo_bfs_shard_loop(C.byref(ops), n + 1, C.byref(depth))
    parts = [None, None]
    dist.all_gather_object(parts, level[:r1 - r0].tolist())
    dist.destroy_process_group()
    q.put((rank, st, depth.value, sum(parts, [])))


def _run_shard_ranks(b):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_shard_rank, args=(r, port, q, b)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=300)
        assert p.exitcode == 0
    return {r: (st, d, lv) for r, st, d, lv in (q.get(timeout=10) for _ in range(2))}


def test_sharded_bfs_two_ranks_gloo(orc, gbo):
    """Two gloo ranks run the library's sharded loop (all-gather of frontier
    words, sum of counts) with the level step restated on the CPU; the
    joined levels are the BFS levels, at two tile widths."""
    csr = gbo.gen_rmat(10, 8, seed=4)
    want, d = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, 5)
    for b in (32, 8):
        res = _run_shard_ranks(b)
        assert res[0][0] == 0 and res[1][0] == 0
        assert res[0][1] == res[1][1] == d
        assert np.array_equal(np.array(res[0][2]), want) and res[0][2] == res[1][2]


def test_shard_loop_agrees_on_a_failed_level(gbo):
    """A rank whose level step fails adds the error mark to the count sum:
    every rank leaves the loop at that level with an error (here one process
    plays both ranks' sums: its own failure and a healthy peer's count)."""
    import ctypes as C

    calls = {"level": 0, "exchange": 0}

    def level_fn(user, lvl, count):
        calls["level"] += 1
        if lvl == 2:
            return 2  # GBO_ERR_CUDA
        count[0] = 10
        return 0

    def allreduce_fn(user, value):
        value[0] = value[0] + 7  # the peer's count
        return 0

    def exchange_fn(user):
        calls["exchange"] += 1
        return 0

    ops = gbo.ShardOps(None, gbo.SHARD_LEVEL_FN(level_fn), gbo.SHARD_ALLREDUCE_FN(allreduce_fn),
                       gbo.SHARD_EXCHANGE_FN(exchange_fn))
    depth = C.c_int(-1)
    st = gbo.lib().gbo_bfs_shard_loop(C.byref(ops), 100, C.byref(depth))
    assert st == 2 and calls == {"level": 3, "exchange": 2} and depth.value == -1
    assert "level 2" in gbo.lib().gbo_last_error().decode()
    # a loop that never converges stops at max_levels
    ops2 = gbo.ShardOps(None, gbo.SHARD_LEVEL_FN(lambda u, l, c: c.__setitem__(0, 1) or 0),
                        gbo.SHARD_ALLREDUCE_FN(lambda u, v: 0), gbo.SHARD_EXCHANGE_FN(lambda u: 0))
    assert gbo.lib().gbo_bfs_shard_loop(C.byref(ops2), 5, C.byref(depth)) == gbo.GBO_ERR_TIMEOUT
