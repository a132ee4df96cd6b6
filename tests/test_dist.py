"""Multi-process paths on the CPU (gloo, world size 2): the benchmark runs
one replica per GPU with no data-path collective; its ranks meet only at the
host barrier and the max-over-ranks reduction of the timed region, and the
reference arm runs on rank 0 alone.  The block-row sharded BFS exchanges
frontier words and counts between ranks (shard.py)."""
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


def _shard_rank(rank, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2")
    sys.path.insert(0, os.path.join(ROOT, "graph-bit-ops_b200"))
    import numpy as np
    import torch
    import torch.distributed as dist

    import gbo
    import shard

    class CpuShard(shard.BfsShard):
        """The shard's level step restated on the CPU (the exchange and the
        loop are the library's own)."""

        def __init__(self, csr, bounds, rank, b):
            super().__init__(csr, bounds, rank, b, device="cpu")
            self.part = shard.shard_csr(csr, self.r0, self.r1)

        def level_step(self, lvl):
            b = self.b
            fw = self.front.numpy().view(np.uint32 if b == 32 else np.uint8).astype(np.uint64)
            onbits = np.zeros(self.nbr_all * b, bool)
            for r in range(b):
                onbits[r::b] = (fw >> np.uint64(b - 1 - r)) & np.uint64(1)
            lv = self.level.numpy()
            nxt = np.zeros(self.nbr * b, bool)
            rp, ci = self.part.rowptr, self.part.colind
            for i in range(self.r1 - self.r0):
                if lv[i] == -1 and onbits[ci[rp[i]:rp[i + 1]]].any():
                    lv[i] = lvl + 1
                    nxt[i] = True
            words = np.zeros(self.nbr, np.uint64)
            for r in range(b):
                words |= nxt[r::b].astype(np.uint64) << np.uint64(b - 1 - r)
            nv = torch.from_numpy(words.astype(np.uint32 if b == 32 else np.uint8).view(
                np.int32 if b == 32 else np.uint8))
            self.next[: self.nbr] = nv
            return int(nxt.sum())

    dist.init_process_group("gloo")
    csr = gbo.gen_rmat(10, 8, seed=4)
    bounds = shard.partition_rows(csr.rowptr, csr.nrows, 2, 32)
    sh = CpuShard(csr, bounds, rank, 32)
    depth = shard.run_distributed(sh, 5)
    parts = [None, None]
    dist.all_gather_object(parts, sh.levels().numpy().tolist())
    dist.destroy_process_group()
    q.put((rank, depth, sum(parts, [])))


def test_sharded_bfs_two_ranks_gloo(orc, gbo):
    """Two gloo ranks run the sharded loop (all-gather of frontier words,
    all-reduce of counts) with the level step restated on the CPU; the
    joined levels are the BFS levels."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_shard_rank, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=300)
        assert p.exitcode == 0
    res = dict((r, (d, lv)) for r, d, lv in (q.get(timeout=10) for _ in range(2)))
    csr = gbo.gen_rmat(10, 8, seed=4)
    want, _ = orc.bfs_csr(csr.rowptr, csr.colind, csr.nrows, 5)
    assert res[0][0] == res[1][0]
    assert np.array_equal(np.array(res[0][1]), want) and res[0][1] == res[1][1]
