"""Benchmark: BFS GTEPS on B2SR (bit-packed BSR) on B200, plus the roofline of
the BFS kernel (the cooperative level loop on 32x32 ROW graphs), the plain
BSR-BMV roofline and a CPU baseline.

Workload (one GPU): BFS from vertex 0 on an R-MAT graph of scale 22 (edge
factor 16, a=0.57 b=0.19 c=0.19, seed 0; symmetrised, deduplicated, no
self-loops), packed as 32x32 B2SR tiles.  A step is one full BFS (levels for
every vertex) with the graph resident in HBM.  GTEPS counts the undirected
edges of the traversed component (sum of reached degrees / 2).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (torchrun, one rank per GPU) runs independent replicas of the same
workload (the reference path does not shard); value = total edges / max time.
"""
from __future__ import annotations

import argparse
import json
import os

# The query server's clients deliver results on streams of their own beside
# the engine's: with CUDA's default 8 hardware queues, 14 client streams
# share queues with the engine, and a client's small copy kernel waits behind
# a whole traversal graph queued ahead of it.  Set before CUDA starts.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "graph-bit-ops_b200"))

SCALE, EDGE_FACTOR, SEED, TILE = 22, 16, 0, 32
RMAT = dict(a=0.57, b=0.19, c=0.19)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=SCALE)
    ap.add_argument("--tile", type=int, default=TILE)
    ap.add_argument("--cpu-samples", type=int, default=3, help="BFS runs timed for cpu_baseline")
    ap.add_argument("--layout", default="row", choices=["row", "col"],
                    help="tile layout of the BFS graph (COL: pull steps read only the frontier's column words)")
    ap.add_argument("--direction", default="auto", choices=["auto", "pull"],
                    help="auto: top-down steps while the frontier is small (graph is symmetric)")
    ap.add_argument("--bfs-loop", default="auto", choices=["auto", "graph", "coop"],
                    help="BFS level loop: loop graph of per-level kernels or one cooperative launch")
    ap.add_argument("--coop-blocks", type=int, default=0, help="cooperative BFS grid (0: sized by the graph)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    ap.add_argument("--nvtx", action="store_true", help="NVTX range 'timed' around the suites' timed loops")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving streams")
    ap.add_argument("--no-permuted", action="store_true", help="skip the degree-ordered variant")
    ap.add_argument("--serve-qps", type=float, default=16000.0, help="offered BFS query rate")
    ap.add_argument("--serve-s", type=float, default=1.5, help="seconds of arrivals per stream")
    ap.add_argument("--serve-slots", type=int, default=1024, help="BFS slots of the served streams' server")
    ap.add_argument("--serve-admit", type=float, default=1.0,
                    help="server BFS admission (free-slot fraction; 1: batch mode, each batch one "
                         "multi-source BFS)")
    ap.add_argument("--tc-graphs", default="mesh,rmat", help="graphs of --workload tc (mesh, rmat)")
    ap.add_argument("--tc-variants", default="input,degree", help="vertex orders of --workload tc")
    ap.add_argument("--tc-tiles", default="8,16,32,64", help="tile widths of --workload tc")
    ap.add_argument("--ms-scale", type=int, default=21, help="R-MAT scale of --workload msbfs")
    ap.add_argument("--ms-ks", default="64,256,1024", help="source counts of --workload msbfs")
    ap.add_argument("--ms-push", type=int, default=-1,
                    help="push threshold of --workload msbfs, new (vertex, source) pairs below which "
                         "a level of k <= 64 pushes (-1: the library default, pull)")
    ap.add_argument("--serve-rates", default="1000,10000,100000",
                    help="offered rates of --workload serve (queries/s, comma-separated)")
    ap.add_argument("--ref-scale", type=int, default=21,
                    help="R-MAT scale of --impl reference --workload refgpu (int32 word offsets of the reference)")
    ap.add_argument("--ref-widths", default="4,8,16,32,64", help="tile widths of the refgpu BMV pairs")
    ap.add_argument("--workload", default="bfs", choices=["bfs", "refgpu"] + list(SUITE),
                    help="bfs: the headline line; the others print one line each for the "
                         "remaining workloads (SSSP/CC/PR on R-MAT 22, TC, MS-BFS, many-graph "
                         "batch, PPR forward/adjoint, served streams)")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Dist:
    """Host-side barrier and max over ranks (gloo); a no-op on one process."""

    def __init__(self, ws):
        self.ws = ws
        if ws > 1:
            import datetime

            import torch.distributed as dist

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
            self.dist = dist

    def barrier(self):
        if self.ws > 1:
            self.dist.barrier()

    def max(self, v: float) -> float:
        if self.ws == 1:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.ws > 1:
            self.dist.destroy_process_group()


def workload_name(scale, tile, layout="row"):
    return (f"BFS from vertex 0, R-MAT scale {scale} edge factor {EDGE_FACTOR} "
            f"(a=0.57,b=0.19,c=0.19, seed {SEED}, symmetrised, deduplicated), B2SR {tile}x{tile}, "
            f"{'column' if layout == 'col' else 'row'}-word tiles")


def traversed_edges(csr, levels):
    deg = np.diff(csr.rowptr).astype(np.int64)
    return int(deg[levels >= 0].sum() // 2)


# --------------------------------------------------------------- roofline
def bfs_level_bytes(rowptr_b, colind_b, levels, nrows, b, row_live, layout="row", csr=None):
    """Algorithmic bytes of each BFS pull step (the words the step must touch).

    Step L reads the block-row offsets, the visited and frontier words, the
    block-column index of every tile in a block row that still has an
    unvisited vertex that can be reached (its row of P has an entry), and --
    only for tiles whose frontier segment is non-empty -- the tile words that
    decide the step: with ROW tiles one b-bit row word per such row, with COL
    tiles one column word per frontier vertex of the segment; it writes the
    next frontier words, visited words of changed rows and one int32 level
    per new vertex.  32x32 ROW tiles carry an occupancy word per tile (read
    with the block-column index); there the step needs only the non-empty
    row words of unvisited rows, counted from the CSR (`csr`) as the distinct
    (row, block column) pairs.
    """
    nbr = len(rowptr_b) - 1
    wb = max(1, b // 8)
    pad = np.full(nbr * b, -2, np.int64)
    pad[:nrows] = levels
    lv = pad.reshape(nbr, b)
    live = np.zeros(nbr * b, bool)
    live[:nrows] = row_live
    live = live.reshape(nbr, b)
    depth = int(levels.max()) + 1
    row_of = np.repeat(np.arange(nbr, dtype=np.int64), np.diff(rowptr_b))
    occ = csr is not None and b == 32 and layout == "row"
    if occ:
        # non-empty row words: distinct (row, block column) pairs of P
        prow = np.repeat(np.arange(nrows, dtype=np.int32), np.diff(csr.rowptr))
        pcol = (csr.colind // b).astype(np.int32)
        first = np.ones(len(pcol), bool)
        first[1:] = (pcol[1:] != pcol[:-1]) | (prow[1:] != prow[:-1])
        prow, pcol = prow[first], pcol[first]
        del first
    out = []
    for L in range(depth):
        unvis = (((lv == -1) | (lv > L)) & live).sum(axis=1)  # reachable unvisited rows
        front_nz = (lv == L).any(axis=1)
        open_row = unvis > 0
        t_open = open_row[row_of]
        t_need = t_open & front_nz[colind_b]
        newv = int((lv == L + 1).sum())
        changed = int(((lv == L + 1).any(axis=1)).sum())
        by = 4 * (nbr + 1) + 2 * wb * nbr + wb * changed + 4 * newv
        by += 4 * int(t_open.sum())
        if occ:
            unv_v = np.zeros(nrows, bool)
            unv_v[:] = (levels == -1) | (levels > L)
            by += 4 * int(t_open.sum())  # occupancy words
            by += wb * int(np.count_nonzero(front_nz[pcol] & unv_v[prow]))
        elif layout == "col":
            fcount = (lv == L).sum(axis=1)  # frontier vertices per block column
            by += wb * int(fcount[colind_b[t_need]].sum())
        else:
            by += wb * int(unvis[row_of[t_need]].sum())
        out.append(by)
    return out


def bfs_push_bytes_rws(csr, levels, L, head=8, long_tail=64):
    """Algorithmic bytes of the cooperative loop's push step at level L over
    the row-word slices: the frontier word of every block row read and one
    frontier word cleared (8 bytes per block row); for every frontier row its
    16-byte tail offsets and its `head` head slots (8 bytes each, sentinels
    included), then every tail entry (8 bytes; a tail longer than
    `long_tail` goes through the push list, 16 bytes more); 4 bytes of level
    per new vertex and 8 bytes (next-frontier and visited words) per changed
    block row.  Visited-word gathers and next-frontier atomics are excluded
    (512 KB vectors that L2 holds), as in the pull model."""
    n = csr.nrows
    nbr = (n + 31) // 32
    front = levels == L
    bc = (csr.colind // 32).astype(np.int64)
    prow = np.repeat(np.arange(n, dtype=np.int64), np.diff(csr.rowptr))
    first = np.ones(len(bc), bool)
    first[1:] = (bc[1:] != bc[:-1]) | (prow[1:] != prow[:-1])
    npairs = np.bincount(prow[first], minlength=n).astype(np.int64)
    tail = np.maximum(npairs - head, 0)[front]
    newv = levels == L + 1
    changed = int(np.count_nonzero(np.pad(newv, (0, nbr * 32 - n)).reshape(nbr, 32).any(axis=1)))
    return (8 * nbr + int(front.sum()) * (16 + 8 * head) + 8 * int(tail.sum())
            + 16 * int(np.count_nonzero(tail > long_tail)) + 4 * int(newv.sum()) + 8 * changed)


def bfs_level_bytes_rws(csr, levels, head=8):
    """Algorithmic bytes of each BFS pull step over the row-word slices of a
    32x32 ROW graph (every row's non-empty row words with their block
    columns, ascending).  Step L reads the visited word and clears one
    frontier word of every block row (8 bytes per block row); for every open
    row (unvisited, with an entry) it reads the 8-byte entries {block
    column, row word} in ascending block column up to and including the
    first whose frontier segment meets the word (all of them when none
    does), plus the 16-byte tail offsets of a row that goes past its first
    `head` entries; it writes the next frontier and visited words of changed
    block rows and one int32 level per new vertex.  Frontier-word gathers
    are excluded, as in the BMV models (a 512 KB vector that L2 holds)."""
    n = csr.nrows
    nbr = (n + 31) // 32
    prow = np.repeat(np.arange(n, dtype=np.int64), np.diff(csr.rowptr))
    pcol = (csr.colind // 32).astype(np.int64)
    first = np.ones(len(pcol), bool)
    first[1:] = (pcol[1:] != pcol[:-1]) | (prow[1:] != prow[:-1])
    pstart = np.flatnonzero(first)
    pr = prow[pstart]
    del prow, pcol, first
    npairs = np.bincount(pr, minlength=n).astype(np.int64)
    rstart = np.concatenate([[0], np.cumsum(npairs)])[:-1]
    pos = np.arange(len(pstart), dtype=np.int64) - rstart[pr]
    has = npairs > 0
    big = np.iinfo(np.int64).max
    out = []
    for L in range(int(levels.max()) + 1):
        open_ = ((levels == -1) | (levels > L)) & has
        newv = levels == L + 1
        changed = int(np.count_nonzero(np.pad(newv, (0, nbr * 32 - n)).reshape(nbr, 32).any(axis=1)))
        by = 8 * nbr + 8 * changed + 4 * int(newv.sum())
        if open_.any():
            hit = np.logical_or.reduceat((levels == L)[csr.colind], pstart)
            key = np.where(hit, pos, big)
            fh = np.full(n, big, np.int64)
            fh[has] = np.minimum.reduceat(key, rstart[has])
            examined = np.where(fh < big, fh + 1, npairs)[open_]
            by += 8 * int(examined.sum()) + 16 * int(np.count_nonzero(examined > head))
        out.append(by)
    return out


def row_word_counts(csr, b=32):
    """Non-empty b-bit row words of every row: its distinct block columns."""
    prow = np.repeat(np.arange(csr.nrows, dtype=np.int64), np.diff(csr.rowptr))
    pcol = (csr.colind // b).astype(np.int64)
    first = np.ones(len(pcol), bool)
    first[1:] = (pcol[1:] != pcol[:-1]) | (prow[1:] != prow[:-1])
    return np.bincount(prow[first], minlength=csr.nrows).astype(np.int64)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(name, algorithmic=None):
    """Per-launch DRAM bytes of a kernel from a committed ncu summary, if any
    (its `traffic_bytes_per_launch:` line).  With `algorithmic` (this run's
    algorithmic bytes per launch) and an `algorithmic_bytes_per_launch:` line
    in the summary, the captured traffic is scaled by their ratio: the
    capture ran a smaller case of the same kernel."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    vals = {}
    with open(p) as f:
        for line in f:
            for key in ("traffic_bytes_per_launch", "algorithmic_bytes_per_launch"):
                if line.startswith(key + ":"):
                    try:
                        vals[key] = float(line.split(":", 1)[1])
                    except ValueError:
                        pass
    t = vals.get("traffic_bytes_per_launch")
    a = vals.get("algorithmic_bytes_per_launch")
    if t is None:
        return None
    if algorithmic is not None and a:
        return t * algorithmic / a
    return t


# ----------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, device):
        self.proc = None
        self.path = os.path.join("/tmp", f"gbo_clocks_{os.getpid()}.csv")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(device),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                t = [x.strip() for x in line.split(",")]
                if len(t) < 8:
                    continue
                try:
                    sm.append(float(t[0]))
                    mx.append(float(t[1]))
                except ValueError:
                    continue
                for nm, val in zip(names, t[4:8]):
                    if val.lower() == "active":
                        reasons.add(nm)
        os.remove(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(mx)) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ------------------------------------------------------------ CPU legs
def cpu_bfs_single(orc, bs, csr, samples):
    """The same CPU BFS on one thread, median of `samples` runs: (GTEPS, seconds)."""
    lv, _ = orc.bfs_b2sr(bs, 0)
    threads = orc.max_threads()
    orc.set_threads(1)
    times = []
    try:
        for _ in range(max(1, samples)):
            t0 = time.perf_counter()
            orc.bfs_b2sr(bs, 0)
            times.append(time.perf_counter() - t0)
    finally:
        orc.set_threads(threads)
    t = float(np.median(times))
    return traversed_edges(csr, lv) / t / 1e9, t


def cpu_bfs(orc, bs, csr, samples):
    """The oracle's port of the reference BFS loop (algorithm/bfs.cu:508-564)
    on B2SR with OpenMP over block rows; returns (GTEPS, seconds, threads,
    levels, depth)."""
    lv, depth = orc.bfs_b2sr(bs, 0)
    edges = traversed_edges(csr, lv)
    times = []
    for _ in range(max(1, samples)):
        t0 = time.perf_counter()
        orc.bfs_b2sr(bs, 0)
        times.append(time.perf_counter() - t0)
    t = float(np.median(times))
    return edges / t / 1e9, t, orc.max_threads(), lv, depth


def bfs_config(args, n, nnz, nblocks, edges, depth, ws):
    """The `config` object of the BFS line, shared by both arms so that the
    same workload is named by the same keys and values."""
    nbr = (n + args.tile - 1) // args.tile
    wb = max(1, args.tile // 8)
    return {"workload": workload_name(args.scale, args.tile, args.layout), "scale": args.scale,
            "tile_bits": args.tile, "layout": args.layout, "nvertices": n, "nnz": int(nnz),
            "nblocks": int(nblocks), "b2sr_gb": (4 * (nbr + 1) + 4 * nblocks + nblocks * args.tile * wb) / 1e9,
            "traversed_edges": int(edges), "bfs_depth": int(depth),
            "l2": "inputs larger than L2 (B2SR tiles far above 126 MB)",
            "parallelism": "replicas" if ws > 1 else "single"}


def run_reference(args, ws, rank):
    """--impl reference: the reference path's CPU restatement (the reference
    has no CPU implementation of its own; its drivers need a GPU and removed
    cuSPARSE APIs), all host threads, same workload, metric and unit.  The
    input graph, the packing and the traversal all come from the oracle, so
    this arm loads no product library."""
    if rank != 0:
        return
    orc = _oracle()
    csr = orc.gen_rmat(args.scale, EDGE_FACTOR, seed=SEED, **RMAT)
    bs = orc.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, args.tile)
    lv, depth = orc.bfs_b2sr(bs, 0)
    edges = traversed_edges(csr, lv)
    for _ in range(args.warmup):
        orc.bfs_b2sr(bs, 0)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        orc.bfs_b2sr(bs, 0)
    dt = (time.perf_counter() - t0) / args.steps
    v = edges / dt / 1e9
    line = {
        "impl": "reference", "metric": "GTEPS", "value": v, "unit": "GTEPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": bfs_config(args, csr.nrows, csr.nnz, bs.nblk, edges, depth, ws),
        "cpu_baseline": {"value": v, "unit": "GTEPS", "cores": orc.max_threads(), "kind": "port",
                         "sample": f"{args.steps} full BFS runs from vertex 0 (oracle port of "
                                   "algorithm/bfs.cu:508-564 on B2SR, OpenMP over block rows)"},
        "e2e": {"value": v, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- serving
def warm_server(gbo, srv, n, slots, seed):
    """Batch mode allocates its level store on the first batch and a
    traversal state (and its captured graph) on the first batch of each
    frontier width: one batch per width (32, 64, ... slots queries) before a
    stream's arrivals start, so that no stream pays that setup."""
    import ctypes

    rng = np.random.default_rng(seed)
    m = 1
    while m <= slots:
        ts = [srv.submit_bfs(int(s)) for s in rng.integers(0, n, m)]
        for t in ts:
            gbo.check(gbo.lib().gbo_server_wait(srv.h, t, None, None, None, ctypes.c_double(300.0)), "warm")
        m = 33 if m == 1 else 2 * m - 1 if m < slots else slots + 1


def serve_stream(gbo, g, n, rate_qps, duration_s, ppr_frac, seed, delivery="host", sample_every=0, slots=64,
                 admit=None):
    """Poisson arrivals of BFS sources and PPR sets (1..64 vertices, Dirichlet
    weights) into the continuous-batching server.  `delivery`: "host" (int32
    levels in host memory, gbo_server_wait), "u8" (byte levels in pinned
    host memory, gbo_server_wait_u8) or "device" (int32 levels in a device
    buffer of the client's, gbo_server_wait_device).  qps = completed
    queries / (last completion - first arrival); latency = submit to result
    in the client's buffer (p50/p99).  With sample_every > 0 every such
    BFS query keeps its result (source, int32 levels) for a parity check.
    In batch mode (admit >= 1) the server is warmed first (warm_server) and
    its counters are reported from after the warm-up."""
    import ctypes
    import queue
    import threading

    rng = np.random.default_rng(seed)
    nq = max(1, int(rate_qps * duration_s))
    gaps = rng.exponential(1.0 / rate_qps, nq)
    kinds = rng.random(nq) < ppr_frac
    qs = []
    for i in range(nq):
        if kinds[i]:
            m = int(rng.integers(1, 65))
            qs.append(("ppr", (rng.choice(n, m, replace=False).astype(np.int32),
                               rng.dirichlet(np.ones(m)).astype(np.float32))))
        else:
            qs.append(("bfs", int(rng.integers(0, n))))
    srv = gbo.Server(g, bfs_slots=slots, ppr_slots=32 if ppr_frac > 0 else 0, alpha=0.85, tol=1e-7)
    if admit is not None:
        srv.set_admission(admit)
    st0 = None
    if admit is not None and admit >= 1.0:
        warm_server(gbo, srv, n, slots, seed + 1000)
        st0 = srv.stats()
    # one queue and consumer pool per kind, so clients waiting on slow PPR
    # results never hold BFS results back (each pool collects in order)
    tq = {"bfs": queue.Queue(), "ppr": queue.Queue()}
    consumers = {"bfs": 14, "ppr": 4 if ppr_frac > 0 else 0}
    lat = {"bfs": [], "ppr": []}
    done_t = []
    samples = []
    lock = threading.Lock()
    t0 = time.perf_counter()
    first_arrival = t0 + gaps[0]

    def producer():
        t = t0
        for i in range(nq):
            t += gaps[i]
            d = t - time.perf_counter()
            if d > 0:
                time.sleep(d)
            kind, arg = qs[i]
            tq[kind].put((i, srv.submit_bfs(arg) if kind == "bfs" else srv.submit_ppr(*arg)))
        for kind, c in consumers.items():
            for _ in range(c):
                tq[kind].put(None)

    def consumer(kind):
        pinned = None
        if delivery == "device":
            buf = gbo.DeviceBuffer(4 * n)
        elif delivery == "u8" and kind == "bfs":
            p = ctypes.c_void_p()
            gbo.check(gbo.lib().gbo_host_alloc(ctypes.byref(p), n), "host_alloc")
            pinned = p.value
        else:
            buf = np.empty(n, np.int32 if kind == "bfs" else np.float32)
        try:
            while True:
                job = tq[kind].get()
                if job is None:
                    return
                i, ticket = job
                if delivery == "device":
                    ms, _ = srv.wait_device(ticket, buf, timeout=300.0)
                elif pinned is not None:
                    _, ms, _ = srv.wait_u8(ticket, timeout=300.0, out=pinned)
                else:
                    _, ms, _ = srv.wait(ticket, kind, timeout=300.0, out=buf)
                tdone = time.perf_counter()
                keep = None
                if sample_every and kind == "bfs" and i % sample_every == 0:
                    if delivery == "device":
                        keep = buf.to_numpy(np.int32, n)
                    elif pinned is not None:
                        b8 = np.ctypeslib.as_array(ctypes.cast(pinned, ctypes.POINTER(ctypes.c_uint8)), (n,))
                        keep = np.where(b8 == 255, -1, b8.astype(np.int32))
                    else:
                        keep = buf.copy()
                with lock:
                    lat[kind].append(ms)
                    done_t.append(tdone)
                    if keep is not None:
                        samples.append((qs[i][1], keep))
        finally:
            if pinned is not None:
                gbo.lib().gbo_host_free(pinned)

    ths = [threading.Thread(target=producer)]
    for kind, c in consumers.items():
        ths += [threading.Thread(target=consumer, args=(kind,)) for _ in range(c)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    st = srv.stats()
    if st0 is not None:
        st = {k: st[k] - st0[k] if k not in ("pending", "in_flight") else st[k] for k in st}
    srv.close()
    span = max(done_t) - first_arrival if done_t else float("nan")
    out = {"offered_qps": rate_qps, "queries": nq, "delivery": delivery, "bfs_slots": slots,
           "admission": "batch mode (warmed)" if st0 is not None else admit, "qps": len(done_t) / span,
           "span_s": span, "rounds": st["rounds"], "kernel_launches": st["kernel_launches"],
           "phase_ms": {k: round(st[k], 1) for k in ("bfs_round_ms", "ppr_round_ms", "retire_ms", "copy_ms",
                                                     "copy_wait_ms", "copy_d2h_ms", "copy_widen_ms")}}
    for k, v in lat.items():
        if v:
            out[f"{k}_p50_ms"] = float(np.percentile(v, 50))
            out[f"{k}_p99_ms"] = float(np.percentile(v, 99))
            out[f"{k}_count"] = len(v)
            if len(lat) > 1 and lat["ppr"]:
                out[f"{k}_qps"] = len(v) / span
    return out, samples


def served_suite(gbo, g, n, plain_ms, rate, dur, check_fn, seed=5, slots=64, admit=None):
    """Capacity of the server with each delivery (a stream offered above it),
    then streams offered at 50 % and 90 % of that capacity (p50/p99 of
    service latency, not of a queue), and a 10 % PPR mix.  Every stream's
    sampled BFS results are checked with check_fn(source, levels)."""
    plain_qps = 1e3 / plain_ms
    res = {"plain_bfs_qps": plain_qps, "qps_definition": "completed queries / (last completion - first arrival)"}
    ok = True
    for delivery, offered in (("device", 2.0 * rate), ("u8", rate), ("host", rate)):
        cap, smp = serve_stream(gbo, g, n, offered, dur, 0.0, seed, delivery, sample_every=97, slots=slots,
                                admit=admit)
        ok = ok and all(check_fn(src, lv) for src, lv in smp)
        cap["vs_plain_bfs_qps"] = cap["qps"] / plain_qps
        res[f"capacity_{delivery}"] = cap
        if delivery == "host":
            continue
        for frac in (0.5, 0.9):
            r, smp = serve_stream(gbo, g, n, frac * cap["qps"], dur, 0.0, seed + 1, delivery, sample_every=97,
                                  slots=slots, admit=admit)
            ok = ok and all(check_fn(src, lv) for src, lv in smp)
            r["vs_plain_bfs_qps"] = r["qps"] / plain_qps
            res[f"{delivery}_{int(frac * 100)}pct"] = r
    mixed, smp = serve_stream(gbo, g, n, rate / 8, dur, 0.1, seed + 2, "u8", sample_every=13, slots=slots,
                              admit=admit)
    ok = ok and all(check_fn(src, lv) for src, lv in smp)
    res["mixed_10pct_ppr"] = mixed
    res["parity"] = {"checked": "every 97th BFS result of each stream (13th of the mix) against gbo_bfs of "
                                "the same source run alone, bit for bit", "equal": bool(ok)}
    return res


# ------------------------------------------------------------- our arm
def run_ours(args, ws, rank, local):
    import gbo

    gbo.check(gbo.lib().gbo_set_device(local), "set_device")
    dist = Dist(ws)
    csr = gbo.gen_rmat(args.scale, EDGE_FACTOR, seed=SEED, **RMAT)
    t0 = time.perf_counter()
    # the symmetrised R-MAT graph may take top-down steps on small frontiers
    flags = gbo.FLAG_SYMMETRIC if args.direction == "auto" else 0
    if args.layout == "col":
        flags |= gbo.FLAG_LAYOUT_COL
    g = gbo.Graph.from_csr(csr, args.tile, flags)
    build_s = time.perf_counter() - t0
    loops = {"auto": gbo.BFS_LOOP_AUTO, "graph": gbo.BFS_LOOP_GRAPH, "coop": gbo.BFS_LOOP_COOP}
    g.set_bfs_loop(loops[args.bfs_loop], args.coop_blocks)
    info = g.info()
    n = csr.nrows
    d_level = gbo.DeviceBuffer(4 * n)

    # levels of the timed workload (compared with the oracle in the CPU leg)
    levels, depth = g.bfs(0)
    edges = traversed_edges(csr, levels)

    clocks = ClockSampler(local)  # samples from the warm-up to the end of the timed runs
    for _ in range(args.warmup):
        g.bfs(0, out=d_level)
    ev0, ev1 = gbo.Event(), gbo.Event()
    dist.barrier()
    gbo.sync()
    ev0.record()
    for _ in range(args.steps):
        g.bfs(0, out=d_level, wait=False)  # queued back to back: the loop runs on the device
    ev1.record()
    gbo.sync()
    dist.barrier()
    ms = ev0.elapsed_ms(ev1) / args.steps
    ms_max = dist.max(ms)
    # per-level times (device clock stamps at every level's end) and kernel
    # launches per BFS, from the same call run once more per step
    step_ms_all, launches = [], 0
    for _ in range(args.steps):
        g.bfs(0, out=d_level)
        st = g.last_run()
        step_ms_all.extend(st["step_ms"])
        launches += st["kernel_launches"]

    # e2e: same call with every step's levels read back into pinned host
    # memory.  Two result buffers and a copy stream: the read-back of step i
    # runs while step i+1 traverses; the copy stream is drained before a
    # buffer is reused and before the closing event.
    d_levels = [d_level, gbo.DeviceBuffer(4 * n)]
    h_levels = [C_pinned(4 * n), C_pinned(4 * n)]
    copy_stream = gbo.Stream()
    g.bfs(0, out=d_levels[1])
    dist.barrier()
    gbo.sync()
    ev0.record()
    for i in range(args.steps):
        g.bfs(0, out=d_levels[i % 2])  # returns when the levels are written
        copy_stream.sync()
        gbo.check(gbo.lib().gbo_memcpy_d2h(h_levels[i % 2].ptr, d_levels[i % 2].ptr, 4 * n,
                                           copy_stream.ptr), "d2h")
    copy_stream.sync()
    ev1.record()
    gbo.sync()
    dist.barrier()
    e2e_ms = dist.max(ev0.elapsed_ms(ev1) / args.steps)

    # the other level loop on the same BFS (b = 32 ROW graphs have both): the
    # loop graph of per-level kernels beside the cooperative launch
    other_loop = None
    if args.tile == 32 and args.layout == "row":
        cur = g.last_run()["kernel_launches"] == 2  # the cooperative form launches 2 kernels
        g.set_bfs_loop(gbo.BFS_LOOP_GRAPH if cur else gbo.BFS_LOOP_COOP, args.coop_blocks)
        for _ in range(3):
            g.bfs(0, out=d_level)
        gbo.sync()
        ev0.record()
        for _ in range(args.steps):
            g.bfs(0, out=d_level, wait=False)
        ev1.record()
        gbo.sync()
        oms = ev0.elapsed_ms(ev1) / args.steps
        olv = g.bfs(0)[0]
        other_loop = {"loop": "graph" if cur else "cooperative", "ms_per_bfs": oms,
                      "gteps": edges / (oms / 1e3) / 1e9, "levels_equal": bool(np.array_equal(olv, levels)),
                      "headline_loop": "cooperative" if cur else "graph"}
        g.set_bfs_loop(loops[args.bfs_loop], args.coop_blocks)

    # pull-only runs of the same BFS (every level a bottom-up step): per-level
    # times beside the direction-optimising ones
    g.set_bfs_direction(False)
    for _ in range(2):
        g.bfs(0, out=d_level)
    auto_step_ms, step_ms_all = step_ms_all, []
    ev0.record()
    for _ in range(args.steps):
        g.bfs(0, out=d_level)
        step_ms_all.extend(g.last_run()["step_ms"])
    ev1.record()
    gbo.sync()
    pull_ms = ev0.elapsed_ms(ev1) / args.steps
    if args.direction == "auto":
        g.set_bfs_direction(True)
    peak, peak_src = load_peaks()
    pull_lvl_ms = np.array(step_ms_all, np.float64).reshape(args.steps, -1).mean(axis=0)
    auto_lvl_ms = np.array(auto_step_ms, np.float64).reshape(args.steps, -1).mean(axis=0)
    rws = args.tile == 32 and args.layout == "row"
    coop = rws and other_loop is not None and other_loop["headline_loop"] == "cooperative"
    rl_launch = None
    if rws:
        # 32x32 ROW graphs traverse their row-word slices; level L pushes iff
        # 0 < |level L| < n/64 (the library's default)
        lvl_bytes = bfs_level_bytes_rws(csr, levels)
        sizes = np.bincount(levels[levels >= 0], minlength=len(lvl_bytes))
        thr = max(1, n // 64) if args.direction == "auto" else 0
        nlv = min(len(lvl_bytes), len(auto_lvl_ms))
        pushed = [thr > 0 and 0 < sizes[L] < thr for L in range(nlv)]
        if coop:
            # one launch (k_bfs_coop) is the whole BFS: every level, pull or push
            for L in range(nlv):
                if pushed[L]:
                    lvl_bytes[L] = bfs_push_bytes_rws(csr, levels, L)
            pull_lv = list(range(nlv))
            rl_bytes = [float(sum(lvl_bytes[:nlv]))]
            rl_ms = [float(np.sum(auto_lvl_ms[:nlv]))]
            rl_launch = {"levels_pushed": [L for L in range(nlv) if pushed[L]]}
            kernel_name = "k_bfs_coop (cooperative BFS loop over row-word slices, one launch per BFS)"
            traffic = load_traffic("k_bfs_coop_rmat20_ncu.md", rl_bytes[0])
        else:
            pull_lv = [L for L in range(nlv) if not pushed[L]]
            rl_bytes = [lvl_bytes[L] for L in pull_lv]
            rl_ms = [float(auto_lvl_ms[L]) for L in pull_lv]
            kernel_name = "k_bfs_pull_rws (BFS pull step over row-word slices, pull levels of the timed runs)"
            traffic = None
        traffic_note = "ncu capture of the same kernel at R-MAT 20 in profiles/, scaled by algorithmic bytes"
    else:
        r = C_void()
        c = C_void()
        gbo.check(gbo.lib().gbo_graph_b2sr(g.h, r.ref(), c.ref(), None), "graph_b2sr")
        rowptr_b = gbo.device_to_numpy(r.value, np.int32, info.nblockrows + 1)
        colind_b = gbo.device_to_numpy(c.value, np.int32, int(info.nblocks))
        lvl_bytes = bfs_level_bytes(rowptr_b, colind_b, levels, n, args.tile, np.diff(csr.rowptr) > 0,
                                    args.layout, csr)
        k = min(len(lvl_bytes), len(pull_lvl_ms))
        pull_lv = list(range(k))
        rl_bytes, rl_ms = lvl_bytes[:k], [float(x) for x in pull_lvl_ms[:k]]
        kernel_name = f"k_bfs_step{'_col' if args.layout == 'col' else ''}<{args.tile}> (BFS pull step, pull-only runs)"
        traffic, traffic_note = None, None
    achieved = sum(rl_bytes) / (sum(rl_ms) / 1e3) / 1e9

    # the BMV primitives, multi-source BFS and the server run on ROW tiles
    g_row = g if args.layout == "row" else gbo.Graph.from_csr(csr, args.tile, gbo.FLAG_SYMMETRIC)

    # plain BSR-BMV count roofline on the same graph (random x, density 0.5)
    x = (np.random.default_rng(0).random(n) < 0.5).astype(np.int32)
    xw = gbo.bits_from_numpy(x, args.tile)
    dx = gbo.DeviceBuffer.from_numpy(xw)
    dy = gbo.DeviceBuffer(4 * n)
    for _ in range(3):
        g_row.bmv_count(dx, dy)
    gbo.sync()
    ev0.record()
    nb = 20
    for _ in range(nb):
        g_row.bmv_count(dx, dy)
    ev1.record()
    gbo.sync()
    bmv_ms = ev0.elapsed_ms(ev1) / nb
    clk = clocks.stop()

    # batched: k sources per multi-source BFS (bit frontier matrix) vs one
    # source per plain BFS, same graph, queries per second
    batched = {}
    ms_sample = None
    rng = np.random.default_rng(3)
    for kq in (64, 1024):
        srcs = rng.integers(0, n, kq).astype(np.int32)
        d_lv = gbo.DeviceBuffer(4 * n * kq)
        g_row.msbfs(srcs, out=d_lv)
        gbo.sync()
        reps = 3
        ev0.record()
        for _ in range(reps):
            g_row.msbfs(srcs, out=d_lv)
        ev1.record()
        gbo.sync()
        mms = ev0.elapsed_ms(ev1) / reps
        batched[f"k{kq}"] = {"ms": mms, "qps": kq / (mms / 1e3),
                            "qps_vs_plain": (kq / mms) / (1.0 / ms)}
        if kq == 1024:  # 16 seeded columns kept for the CPU leg's parity check
            ms_cols = np.random.default_rng(17).choice(kq, 16, replace=False)
            ms_sample = (srcs[ms_cols], ms_columns(gbo, d_lv, n, kq, ms_cols))
        d_lv.free()

    # permuted variant (reported beside the headline, never as it): the same
    # graph relabelled by descending degree, BFS from vertex 0's new label
    permuted = None
    if not args.no_permuted and args.layout == "row":
        t0 = time.perf_counter()
        gp = gbo.Graph.from_csr(csr, args.tile, gbo.FLAG_SYMMETRIC | gbo.FLAG_DEGREE_ORDER)
        pbuild = time.perf_counter() - t0
        perm = gp.permutation()
        plv, _ = gp.bfs(int(perm[0]))
        if not np.array_equal(plv[perm], levels):
            raise SystemExit("degree-ordered BFS levels differ from the headline BFS")
        pbuf = gbo.DeviceBuffer(4 * n)
        for _ in range(args.warmup):
            gp.bfs(int(perm[0]), out=pbuf)
        gbo.sync()
        pst = []
        ev0.record()
        for _ in range(args.steps):
            gp.bfs(int(perm[0]), out=pbuf)
            pst.append(gp.last_run()["step_ms"])
        ev1.record()
        gbo.sync()
        pms = ev0.elapsed_ms(ev1) / args.steps
        permuted = {"workload": "the same BFS on the graph relabelled by descending degree",
                    "gteps": edges / (pms / 1e3) / 1e9, "ms_per_bfs": pms,
                    "nblocks": int(gp.info().nblocks), "relabel_and_pack_s": pbuild,
                    "levels_ms": [float(v) for v in np.array(pst).mean(axis=0)]}
        pbuf.free()
        gp.free()

    # served: Poisson query streams into the continuous-batching server
    served = {}
    if not args.no_serve:
        alone = gbo.DeviceBuffer(4 * n)

        def same_as_alone(src, lv):
            g_row.bfs(int(src), out=alone)
            return bool(np.array_equal(alone.to_numpy(np.int32, n), lv))

        served = served_suite(gbo, g_row, n, ms, args.serve_qps, args.serve_s, same_as_alone,
                              slots=args.serve_slots, admit=args.serve_admit)
        alone.free()
    wb = max(1, args.tile // 8)
    bmv_bytes = (int(info.nblocks) * (args.tile * args.tile // 8 + 4) + 4 * (info.nblockrows + 1)
                 + wb * info.nblockcols + 4 * n)
    bmv_gbs = bmv_bytes / (bmv_ms / 1e3) / 1e9

    gteps = ws * edges / (ms_max / 1e3) / 1e9
    line = {
        "metric": "GTEPS", "value": gteps, "unit": "GTEPS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": bfs_config(args, n, csr.nnz, int(info.nblocks), edges, depth, ws),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "traffic_source": traffic_note if traffic is not None else None,
                     "kernel": kernel_name, "peak_source": peak_src,
                     "levels": pull_lv, "launch": rl_launch,
                     "algorithmic_bytes_per_launch": float(np.mean(rl_bytes)),
                     "ms_per_launch": float(np.mean(rl_ms)),
                     # the DRAM traffic (scaled capture) over the same time:
                     # how busy HBM is, beside the algorithmic fraction
                     "traffic_frac": (traffic / (float(np.mean(rl_ms)) / 1e3) / 1e9 / peak
                                      if traffic is not None else None)},
        "e2e": {"value": ws * edges / (e2e_ms / 1e3) / 1e9, "unit": "GTEPS",
                "h2d_bytes_per_step": 4, "d2h_bytes_per_step": 4 * n,
                "overlap": "read-back of step i on a copy stream during step i+1 (two level buffers)"},
        "gpu_launches": int(launches),
        "clocks": clk,
        "bmv_count": {"achieved_gbs": bmv_gbs, "frac": bmv_gbs / peak, "ms": bmv_ms,
                      "algorithmic_bytes": bmv_bytes, "gteps": csr.nnz / (bmv_ms / 1e3) / 1e9},
        "batched_bfs": dict(batched, plain_qps=1e3 / ms),
        "served": served,
        "direction": args.direction,
        "bfs_loop": other_loop["headline_loop"] if other_loop else "graph",
        "other_loop": other_loop,
        "levels_ms": [float(v) for v in auto_lvl_ms],
        "levels_gb": [b / 1e9 for b in lvl_bytes],
        "pull_only": {"ms_per_bfs": pull_ms, "gteps": edges / (pull_ms / 1e3) / 1e9,
                      "levels_ms": [float(v) for v in pull_lvl_ms]},
        "graph_build_s": build_s,
        "permuted_variant": permuted,
    }
    if rank == 0 and ws == 1 and not args.no_cpu:
        # CPU leg: the oracle's port of the reference BFS loop, timed, and its
        # levels (plus an independent queue BFS on the CSR) compared with the
        # GPU's levels of the timed workload
        orc = _oracle()
        bs = orc.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, args.tile)
        v, t, cores, lv_port, d_port = cpu_bfs(orc, bs, csr, args.cpu_samples)
        v1, t1 = cpu_bfs_single(orc, bs, csr, max(3, args.cpu_samples))
        if ms_sample is not None:
            ok = all(np.array_equal(col, orc.bfs_b2sr(bs, int(src))[0])
                     for src, col in zip(ms_sample[0], ms_sample[1].T))
            line["batched_bfs"]["parity"] = {
                "checked": "16 seeded columns of the k = 1024 multi-source BFS against one oracle BFS each",
                "equal": bool(ok)}
        del bs
        lv_q, d_q = orc.bfs_csr(csr.rowptr, csr.colind, n, 0)
        line["cpu_baseline"] = {"value": v, "unit": "GTEPS", "cores": cores, "kind": "port",
                                "sample": f"{args.cpu_samples} full BFS runs from vertex 0 "
                                          f"(median {t:.2f} s), oracle port of algorithm/bfs.cu:508-564",
                                "single_thread": {"value": v1, "unit": "GTEPS", "seconds": t1,
                                                  "samples": max(3, args.cpu_samples)}}
        line["parity"] = {
            "checked": f"int32 BFS levels of all {n} vertices from gbo_bfs against the oracle's port of "
                       "algorithm/bfs.cu:508-564 on B2SR and against a queue BFS on the CSR",
            "equal": bool(np.array_equal(levels, lv_port) and np.array_equal(levels, lv_q)
                          and depth == d_port == d_q),
            "mismatched_vertices": int(np.count_nonzero(levels != lv_q))}
    else:
        line["parity"] = {"checked": False, "why": "CPU leg skipped (--no-cpu or N > 1)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if g_row is not g:
        g_row.free()
    g.free()
    dist.close()


class C_void:
    def __init__(self):
        import ctypes

        self._v = ctypes.c_void_p()

    def ref(self):
        import ctypes

        return ctypes.byref(self._v)

    @property
    def value(self):
        return self._v.value


class C_pinned:
    def __init__(self, nbytes):
        import ctypes

        import gbo

        p = ctypes.c_void_p()
        gbo.check(gbo.lib().gbo_host_alloc(ctypes.byref(p), nbytes), "host_alloc")
        self.ptr = p.value

    def __del__(self):
        try:
            import gbo

            gbo.lib().gbo_host_free(self.ptr)
        except Exception:
            pass


# ----------------------------------------------------------------- suite
# One JSON line per workload, same keys as the headline where they apply.
# Device time by CUDA events around the public C-ABI calls (outputs in
# preallocated device buffers; each call ends with its host-visible result
# such as the iteration count, as a user sees it).  CPU figures are the
# oracle's OpenMP restatement on one bounded sample.


class _Nvtx:
    """An NVTX range named "timed" around a suite's timed loop when --nvtx
    is given (so that ncu --nvtx --nvtx-include timed/ selects its launches,
    whole CUDA graphs included); nothing otherwise."""
    on = False

    def __enter__(self):
        if _Nvtx.on:
            import torch.cuda.nvtx as nv
            nv.range_push("timed")
        return self

    def __exit__(self, *exc):
        if _Nvtx.on:
            import torch.cuda.nvtx as nv
            nv.range_pop()
        return False


def _timed(gbo, fn, steps, warmup):
    for _ in range(warmup):
        fn()
    gbo.sync()
    e0, e1 = gbo.Event(), gbo.Event()
    with _Nvtx():
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        gbo.sync()
    return e0.elapsed_ms(e1) / steps


def _cpu(fn, samples=1):
    ts = []
    for _ in range(samples):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts))


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    return oracle


def _line(metric, value, unit, hib, ms, args, config, **extra):
    d = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
         "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": hib, "scaling": "weak",
         "vs_baseline": None, "data": "synthetic", "config": config}
    d.update(extra)
    print(json.dumps(d), flush=True)


def _bmv_bytes(info, b, n, vec_bytes):
    wb = max(1, b // 8)
    return info.nblocks * (b * wb + 4) + 4 * (info.nblockrows + 1) + vec_bytes


def suite_config2(args, which):
    """SSSP, CC and PageRank (20 iterations) on the headline R-MAT 22 graph."""
    import ctypes as C

    import gbo

    orc = _oracle()
    csr = gbo.gen_rmat(args.scale, EDGE_FACTOR, seed=SEED, **RMAT)
    g = gbo.Graph.from_csr(csr, args.tile, gbo.FLAG_SYMMETRIC)  # symmetrised R-MAT
    info = g.info()
    n = csr.nrows
    lv, depth = g.bfs(0)
    edges = traversed_edges(csr, lv)
    cfg = {"workload": "", "scale": args.scale, "tile_bits": args.tile, "nvertices": n,
           "nnz": csr.nnz, "nblocks": int(info.nblocks),
           "l2": "inputs larger than L2 (B2SR tiles far above 126 MB)"}
    buf = gbo.DeviceBuffer(4 * n)
    it = C.c_int(0)
    peak, psrc = load_peaks()
    bs = orc.pack(csr.rowptr, csr.colind, n, n, args.tile) if not args.no_cpu else None
    if which == "sssp":
        ms = _timed(gbo, lambda: gbo.check(gbo.lib().gbo_sssp_unit(g.h, 0, buf.ptr, C.byref(it), None)),
                    args.steps, args.warmup)
        cfg["workload"] = f"unit-weight SSSP from vertex 0 (min-plus BMV), R-MAT scale {args.scale}"
        extra = {"iterations": it.value, "traversed_edges": edges, "dtype": "u32"}
        if bs is not None:
            got = buf.to_numpy(np.uint32, n)
            res = {}
            t = _cpu(lambda: res.update(d=orc.sssp_b2sr(bs, 0)[0]))
            extra["cpu_baseline"] = {"value": edges / t / 1e9, "unit": "GTEPS", "cores": orc.max_threads(),
                                     "kind": "port", "sample": "1 SSSP from vertex 0 (sssp.cu:420-470 port)"}
            extra["parity"] = {"checked": f"uint32 distances of all {n} vertices against the oracle's "
                                          "min-plus SSSP port (sssp.cu:420-470)",
                               "equal": bool(np.array_equal(got, res["d"]))}
        _line("GTEPS", edges / (ms / 1e3) / 1e9, "GTEPS", True, ms, args, cfg, **extra)
    elif which == "cc":
        ms = _timed(gbo, lambda: gbo.check(gbo.lib().gbo_cc(g.h, buf.ptr, C.byref(it), None)),
                    args.steps, args.warmup)
        und = csr.nnz // 2
        cfg["workload"] = f"connected components (FastSV, min label), R-MAT scale {args.scale}"
        extra = {"iterations": it.value, "undirected_edges": und, "dtype": "i32"}
        if bs is not None:
            got = buf.to_numpy(np.int32, n)
            res = {}
            t = _cpu(lambda: res.update(lab=orc.cc(csr.rowptr, csr.colind, n)))
            extra["cpu_baseline"] = {"value": und / t / 1e9, "unit": "GTEPS", "cores": orc.max_threads(),
                                     "kind": "port", "sample": "1 CC run (label propagation, min id)"}
            bad, ncomp = orc.verify_cc(csr.rowptr, csr.colind, n, got)
            extra["parity"] = {"checked": f"int32 labels of all {n} vertices against the oracle's minimum "
                                          "vertex id per component, and SimpleVerifyCc (cc.cu:21-60)",
                               "equal": bool(np.array_equal(got, res["lab"]) and bad == 0),
                               "components": ncomp}
        _line("GTEPS", und / (ms / 1e3) / 1e9, "GTEPS", True, ms, args, cfg, **extra)
    else:
        iters = 20
        ms = _timed(gbo, lambda: gbo.check(gbo.lib().gbo_pagerank(g.h, C.c_float(0.85), iters, C.c_float(-1.0),
                                                                   buf.ptr, C.byref(it), None)),
                    args.steps, args.warmup)
        st = g.last_run()
        step = float(np.mean(st["step_ms"])) if st["step_ms"] else ms / iters
        if args.tile == 32:
            # row-word slices: every non-empty row word once with its block
            # column (8 bytes), the tail offsets of rows past the head, and
            # per vertex the iterate read, its 1/deg, and the two outputs
            # written (16 bytes); the gathered p/deg words are excluded (a
            # 16 MB vector that L2 holds)
            words = row_word_counts(csr)
            by = 8 * int(words.sum()) + 16 * int(np.count_nonzero(words > 8)) + 16 * n
            kname = "k_pr_step_rws (PageRank iteration over row-word slices)"
        else:
            by = _bmv_bytes(info, args.tile, n, 4 * n * 5)  # p/deg gathered, p, D^-1 read; p', p'/deg written
            kname = "k_pr_step (PageRank iteration, semiring BMV + update)"
        cfg["workload"] = f"PageRank alpha 0.85, 20 iterations, fp32 values / fp64 sums, R-MAT scale {args.scale}"
        extra = {"iterations": it.value, "dtype": "f32",
                 "roofline": {"bound": "hbm", "achieved": by / (step / 1e3) / 1e9, "peak": peak,
                              "unit": "GB/s", "frac": by / (step / 1e3) / 1e9 / peak,
                              "traffic": (load_traffic("k_pr_step_rws_rmat20_ncu.md", by)
                                          if args.tile == 32 else None),
                              "kernel": kname, "peak_source": psrc,
                              "algorithmic_bytes_per_launch": by, "ms_per_launch": step}}
        if bs is not None:
            got = buf.to_numpy(np.float32, n).astype(np.float64)
            outdeg = np.bincount(csr.colind, minlength=n).astype(np.int32)
            t = _cpu(lambda: orc.pagerank_b2sr_f32(bs, outdeg, 0.85, iters, -1.0))
            extra["cpu_baseline"] = {"value": iters * csr.nnz / t / 1e9, "unit": "GTEPS",
                                     "cores": orc.max_threads(), "kind": "port",
                                     "sample": "20 PageRank iterations (pr.cu:449-513 port)"}
            ref, _ = orc.pagerank_f64(csr.rowptr, csr.colind, n, outdeg, 0.85, iters, -1.0)
            rel = float(np.abs(got - ref).sum() / np.abs(ref).sum())
            extra["parity"] = {"checked": "20-iteration PageRank vector against the oracle's fp64 PageRank "
                                          "(pr.cu:449-513 recurrence), relative L1, tolerance 1e-5",
                               "rel_l1": rel, "equal": bool(rel <= 1e-5)}
        _line("GTEPS", iters * csr.nnz / (ms / 1e3) / 1e9, "GTEPS", True, ms, args, cfg, **extra)
    g.free()


def suite_tc(args):
    """Triangle counting: king mesh 4096^2 and R-MAT 20 (seed 1), every tile
    width timed in input vertex order and relabelled by descending degree
    (the count is the same); the fastest combination is the tuned choice."""
    import gbo

    orc = _oracle()
    graphs = {"mesh": lambda: ("king mesh 4096x4096", gbo.gen_king_mesh(4096), 4 * 4095 ** 2),
              "rmat": lambda: ("R-MAT scale 20 ef16 seed 1", gbo.gen_rmat(20, 16, seed=1, **RMAT), None)}
    orders = {"input": gbo.FLAG_LOWER, "degree": gbo.FLAG_LOWER | gbo.FLAG_DEGREE_ORDER}
    for key in args.tc_graphs.split(","):
        name, csr, known = graphs[key]()
        table = {}
        count = None
        for order in args.tc_variants.split(","):
            flags = orders[order]
            for b in (int(t) for t in args.tc_tiles.split(",")):
                t0 = time.perf_counter()
                g = gbo.Graph.from_csr(csr, b, flags)
                build_s = time.perf_counter() - t0
                c = g.tc()
                if count is None:
                    count = c
                if c != count or (known is not None and c != known):
                    raise SystemExit(f"TC mismatch on {name} ({order}, b={b}): {c}")
                ms = _timed(gbo, g.tc, args.steps, args.warmup)
                table[f"{order}/b{b}"] = {"ms": ms, "nblocks_L": int(g.info().nblocks), "build_s": build_s}
                g.free()
        best = min(table, key=lambda k: table[k]["ms"])
        ms = table[best]["ms"]
        model_best, _ = gbo.tune_tile_width(csr, gbo.TUNE_TC, gbo.TUNE_MODEL)
        lower_edges = csr.nnz // 2
        extra = {"triangles": count, "tile_table": table, "best": best, "model_tile_input_order": model_best,
                 "dtype": "u64"}
        if not args.no_cpu:
            res = {}
            t = _cpu(lambda: res.update(n=orc.tc_csr(csr.rowptr, csr.colind, csr.nrows)))
            extra["cpu_baseline"] = {"value": lower_edges / t / 1e9, "unit": "G lower edges/s",
                                     "cores": orc.max_threads(), "kind": "port",
                                     "sample": "1 full count (sorted-adjacency intersection on L)"}
            extra["parity"] = {"checked": "uint64 triangle count of every tile width and vertex order against "
                                          "the oracle's sorted-adjacency count"
                                          + (" and the closed form 4(n-1)^2" if known is not None else ""),
                               "oracle": res["n"], "equal": bool(count == res["n"])}
        _line("G lower edges/s", lower_edges / (ms / 1e3) / 1e9, "G lower edges/s", True, ms, args,
              {"workload": f"triangle count (masked B2SR SpGEMM on L), {name}", "nvertices": csr.nrows,
               "nnz": csr.nnz}, **extra)


def ms_columns(gbo, out, n, k, cols, rows=65536):
    """Columns `cols` of an (n, k) int32 level matrix on the device, read
    back in row chunks: an (n, len(cols)) array."""
    res = np.empty((n, len(cols)), np.int32)
    for r0 in range(0, n, rows):
        m = min(rows, n - r0)
        chunk = np.empty((m, k), np.int32)
        gbo.check(gbo.lib().gbo_memcpy_d2h(chunk.ctypes.data, out.ptr + 4 * r0 * k, chunk.nbytes, None), "d2h")
        gbo.check(gbo.lib().gbo_stream_sync(None), "sync")
        res[r0:r0 + m] = chunk[:, cols]
    return res


def _ms_edges(gbo, out, deg, n, k, rows=65536):
    """Traversed undirected edges summed over the k columns of an (n, k)
    int32 level matrix on the device, read back in row chunks."""
    tot = np.zeros(k, np.float64)
    degf = deg.astype(np.float64)
    for r0 in range(0, n, rows):
        m = min(rows, n - r0)
        chunk = np.empty((m, k), np.int32)
        gbo.check(gbo.lib().gbo_memcpy_d2h(chunk.ctypes.data, out.ptr + 4 * r0 * k, chunk.nbytes, None), "d2h")
        gbo.check(gbo.lib().gbo_stream_sync(None), "sync")
        tot += degf[r0:r0 + m] @ (chunk >= 0)
    return int(tot.sum()) // 2


def suite_msbfs(args):
    """Multi-source BFS on R-MAT 21 (seed 2; --ms-scale), k = 64/256/1024
    sources (seed 3; --ms-ks), queries per second against one plain BFS per
    source."""
    import gbo

    csr = gbo.gen_rmat(args.ms_scale, 16, seed=2, **RMAT)
    g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_SYMMETRIC)
    n = csr.nrows
    rng = np.random.default_rng(3)
    d_level = gbo.DeviceBuffer(4 * n)
    srcs_plain = rng.integers(0, n, 16).astype(np.int32)
    plain_ms = np.mean([_timed(gbo, lambda s=int(s): g.bfs(s, out=d_level), 1, 1) for s in srcs_plain])
    if args.ms_push >= 0:  # after the plain runs, which keep their own default
        g.set_bfs_direction(True, args.ms_push)
    res = {}
    deg = np.diff(csr.rowptr).astype(np.int64)
    ks = [int(k) for k in args.ms_ks.split(",")]
    for k in ks:
        srcs = rng.integers(0, n, k).astype(np.int32)
        out = gbo.DeviceBuffer(4 * n * k)
        ms = _timed(gbo, lambda: g.msbfs(srcs, out=out), max(1, args.steps // 2), args.warmup)
        levels_ms = [round(x, 3) for x in g.last_run()["step_ms"]]
        edges = _ms_edges(gbo, out, deg, n, k)
        res[k] = {"ms": ms, "qps": k / (ms / 1e3), "gteps_x_k": edges / (ms / 1e3) / 1e9,
                  "speedup_vs_plain": (k / (ms / 1e3)) / (1e3 / plain_ms), "levels_ms": levels_ms}
        if not args.no_cpu:
            cols = np.random.default_rng(100 + k).choice(k, min(k, 16), replace=False)
            got = ms_columns(gbo, out, n, k, cols)
            orc = _oracle()
            ok = all(np.array_equal(got[:, i], orc.bfs_csr(csr.rowptr, csr.colind, n, int(srcs[c]))[0])
                     for i, c in enumerate(cols))
            res[k]["parity"] = {"checked": f"{len(cols)} seeded columns against one oracle queue BFS each",
                                "equal": bool(ok)}
        del out
    best = res[max(ks)]
    _line("qps", best["qps"], "queries/s", True, best["ms"], args,
          {"workload": f"multi-source BFS, R-MAT scale {args.ms_scale} ef16 seed 2, k random sources "
                       "(seed 3), B2SR 32",
           "nvertices": n, "nnz": csr.nnz},
          dtype="u32", by_k=res, plain_qps=1e3 / plain_ms, ms_push=args.ms_push,
          parity=({"checked": "16 seeded columns per k against one oracle queue BFS each",
                   "equal": all(r["parity"]["equal"] for r in res.values())}
                  if not args.no_cpu else {"checked": False}))
    g.free()


def suite_batch(args):
    """10,000 ER graphs (n log-uniform in [32, 65536], average degree 8,
    seeds 1000+i) as one block-diagonal B2SR: one multi-seed BFS (vertex 0 of
    every graph) against one BFS per graph on its own handle, at the tile
    width the tuner's byte model picks and at 32x32 (row-word slices and the
    cooperative loop), the faster of the two reported."""
    import gbo

    count = 10000
    t0 = time.perf_counter()
    csr, off = gbo.gen_er_batch(count, 32, 65536, 8.0, 1000)
    gen_s = time.perf_counter() - t0
    b_model, tune_cost = gbo.tune_tile_width(csr, gbo.TUNE_BFS, gbo.TUNE_MODEL)  # bytes model
    n = csr.nrows
    seeds = off[:-1].astype(np.int32)
    rp = csr.rowptr
    ci = csr.colind
    sample = np.random.default_rng(7).choice(count, 100, replace=False)
    runs = {}
    for b in sorted({b_model, 32}):
        g = gbo.Graph.from_csr(csr, b, gbo.FLAG_SYMMETRIC)
        d_level = gbo.DeviceBuffer(4 * n)
        ms = _timed(gbo, lambda: g.bfs_multi(seeds, out=d_level), args.steps, args.warmup)
        nblk = int(g.info().nblocks)
        g.free()
        union_levels = d_level.to_numpy(np.int32, n)
        d_level.free()
        # one graph per handle and per BFS call, on a sample of 100 graphs
        per, checked = [], []
        for i in sample:
            lo, hi = int(off[i]), int(off[i + 1])
            sub_rp = (rp[lo:hi + 1] - rp[lo]).astype(np.int32)
            sub_ci = (ci[rp[lo]:rp[hi]] - lo).astype(np.int32)
            sub = gbo.Csr(sub_rp, sub_ci, hi - lo, hi - lo)
            gs = gbo.Graph.from_csr(sub, b, gbo.FLAG_SYMMETRIC)
            buf = gbo.DeviceBuffer(4 * (hi - lo))
            per.append(_timed(gbo, lambda: gs.bfs(0, out=buf), 3, 1))
            gs.free()
            if not args.no_cpu:
                want, _ = _oracle().bfs_csr(sub_rp, sub_ci, hi - lo, 0)
                checked.append(bool(np.array_equal(union_levels[lo:hi], want)))
        runs[b] = {"ms": ms, "graphs_per_s": count / (ms / 1e3), "nblocks": nblk,
                   "one_by_one_graphs_per_s": 1e3 / float(np.mean(per)),
                   "parity": ({"checked": "levels of 100 seeded graphs of the union against one oracle queue BFS "
                                          "per graph", "equal": all(checked)} if checked else {"checked": False})}
    b = min(runs, key=lambda k: runs[k]["ms"])
    r = runs[b]
    _line("graphs/s", r["graphs_per_s"], "graphs/s", True, r["ms"], args,
          {"workload": "BFS from vertex 0 of each of 10000 ER graphs (n log-uniform 32..65536, avg degree 8, "
                       "seeds 1000+i) packed block-diagonally as one B2SR graph",
           "tile_bits": b, "tuner_model_pick": b_model,
           "tuner_bytes": {k: (v if np.isfinite(v) else None) for k, v in tune_cost.items()},
           "nvertices": n, "nnz": csr.nnz, "nblocks": r["nblocks"], "generate_s": gen_s},
          dtype="bits", one_by_one_graphs_per_s=r["one_by_one_graphs_per_s"],
          speedup=r["graphs_per_s"] / r["one_by_one_graphs_per_s"], by_tile=runs,
          parity=r["parity"] if all(x["parity"].get("equal", True) for x in runs.values()) else
          {"checked": "every width", "equal": False})


def suite_ppr(args):
    """PPR forward and adjoint on R-MAT 20: v Dirichlet over a random 1 % of
    vertices (seed 4), w ~ N(0,1) (seed 5), alpha 0.85, tol 1e-7; gradient
    checked by central differences along 64 random directions."""
    import ctypes as C

    import gbo

    csr = gbo.gen_rmat(20, 16, seed=1, **RMAT)
    n = csr.nrows
    g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_SYMMETRIC)  # adjoint gathers over P = P^T
    rng = np.random.default_rng(4)
    idx = rng.choice(n, n // 100, replace=False)
    v = np.zeros(n)
    v[idx] = rng.dirichlet(np.ones(len(idx)))
    w = np.random.default_rng(5).standard_normal(n)
    dv = gbo.DeviceBuffer.from_numpy(v.astype(np.float32))
    dw = gbo.DeviceBuffer.from_numpy(w.astype(np.float32))
    dp = gbo.DeviceBuffer(4 * n)
    dg = gbo.DeviceBuffer(4 * n)
    it_f, it_b = C.c_int(0), C.c_int(0)
    fwd = _timed(gbo, lambda: gbo.check(gbo.lib().gbo_ppr_forward(g.h, dv.ptr, C.c_float(0.85), C.c_float(1e-7),
                                                                   1000, dp.ptr, C.byref(it_f), None)),
                 args.steps, args.warmup)
    bwd = _timed(gbo, lambda: gbo.check(gbo.lib().gbo_ppr_backward(g.h, dw.ptr, C.c_float(0.85), C.c_float(1e-7),
                                                                    1000, dg.ptr, C.byref(it_b), None)),
                 args.steps, args.warmup)
    grad = dg.to_numpy(np.float32, n).astype(np.float64)
    fwd_p = dp.to_numpy(np.float32, n).astype(np.float64)
    parity = {"checked": False}
    if not args.no_cpu:
        orc = _oracle()
        outdeg = np.bincount(csr.colind, minlength=n).astype(np.int32)
        p_ref, _ = orc.ppr_f64(csr.rowptr, csr.colind, n, outdeg, v, 0.85, 1e-13)
        g_ref, _ = orc.ppr_adjoint_f64(csr.rowptr, csr.colind, n, outdeg, w, 0.85, 1e-13)
        rf = float(np.abs(fwd_p - p_ref).sum() / np.abs(p_ref).sum())
        rb = float(np.abs(grad - g_ref).sum() / np.abs(g_ref).sum())
        parity = {"checked": "PPR vector and gradient against the oracle's fp64 forward and adjoint solves "
                             "(tol 1e-13), relative L1, tolerance 1e-5",
                  "forward_rel_l1": rf, "gradient_rel_l1": rb, "equal": bool(rf <= 1e-5 and rb <= 1e-5)}
    errs = []
    for _ in range(64):
        d = np.zeros(n)
        d[idx] = rng.standard_normal(len(idx))
        pp, _ = g.ppr_forward((v + 1e-3 * d).astype(np.float32), 0.85, 1e-9, 2000)
        pm, _ = g.ppr_forward((v - 1e-3 * d).astype(np.float32), 0.85, 1e-9, 2000)
        fd = (w @ pp.astype(np.float64) - w @ pm.astype(np.float64)) / 2e-3
        errs.append(abs(fd - grad @ d) / max(1.0, abs(fd)))
    _line("ms", fwd + bwd, "ms per forward+adjoint", False, fwd + bwd, args,
          {"workload": "PPR forward + adjoint, R-MAT scale 20 seed 1, v on 1% of vertices, alpha 0.85, tol 1e-7",
           "nvertices": n, "nnz": csr.nnz},
          dtype="f32", forward_ms=fwd, forward_iters=it_f.value, backward_ms=bwd, backward_iters=it_b.value,
          fd_directions=64, fd_max_rel_err=float(max(errs)), parity=parity)
    g.free()


def suite_serve(args):
    """Poisson arrivals at 1k, 10k and 100k queries/s into the continuous
    batching server (R-MAT 21 seed 2, B2SR 32): 90 % BFS sources, 10 % PPR
    sets of 1-64 vertices; achieved rate and p50/p99 latency."""
    import gbo

    csr = gbo.gen_rmat(21, 16, seed=2, **RMAT)
    n = csr.nrows
    g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_SYMMETRIC)  # symmetrised R-MAT: the plain BFS may push
    # plain per-query kernels on the same graph and GPU: one BFS per source,
    # one PPR forward solve per personalization set (same tolerance)
    rng = np.random.default_rng(13)
    buf = gbo.DeviceBuffer(4 * n)
    bfs_ms = float(np.mean([_timed(gbo, lambda s=int(s): g.bfs(s, out=buf), 2, 1)
                            for s in rng.integers(0, n, 8)]))
    import ctypes as C

    it = C.c_int(0)
    ppr_ms = []
    for _ in range(3):
        m = int(rng.integers(1, 65))
        v = np.zeros(n, np.float32)
        v[rng.choice(n, m, replace=False)] = rng.dirichlet(np.ones(m))
        dv = gbo.DeviceBuffer.from_numpy(v)
        ppr_ms.append(_timed(gbo, lambda: gbo.check(gbo.lib().gbo_ppr_forward(
            g.h, dv.ptr, C.c_float(0.85), C.c_float(1e-7), 1000, buf.ptr, C.byref(it), None)), 1, 1))
    plain = {"bfs_qps": 1e3 / bfs_ms, "ppr_qps": 1e3 / float(np.mean(ppr_ms)), "ppr_iterations": it.value}
    out = {}
    rates = [float(r) for r in args.serve_rates.split(",")]
    for rate in rates:
        r, _ = serve_stream(gbo, g, n, rate, min(args.serve_s, 2e4 / rate), 0.1, 11, "u8", slots=args.serve_slots,
                            admit=args.serve_admit)
        r["bfs_vs_plain"] = r.get("bfs_qps", 0.0) / plain["bfs_qps"]
        r["ppr_vs_plain"] = r.get("ppr_qps", 0.0) / plain["ppr_qps"]
        out[int(rate)] = r
    top = out[int(rates[len(rates) // 2])]
    _line("qps", top["qps"], "queries/s", True, 1e3 / max(top["qps"], 1e-9), args,
          {"workload": "served BFS + PPR queries, Poisson arrivals, R-MAT scale 21 seed 2, B2SR 32",
           "nvertices": n, "nnz": csr.nnz}, dtype="u32", plain=plain, by_rate=out)
    g.free()


def suite_spgemm(args):
    """Unmasked binary products: C = L L^T (benchmark-bsrbmm.cu's check) on
    the king mesh 1024^2 and R-MAT 14 (seed 1): the sparse-output product
    (both passes, int64 offsets, int32 columns and counts) and the total of
    A B, against the oracle's CPU product on the same graphs."""
    import ctypes as C

    import gbo

    oracle = _oracle()
    res = {}
    for name, csr in (("mesh1024", gbo.gen_king_mesh(1024)), ("rmat14", gbo.gen_rmat(14, 16, seed=1, **RMAT))):
        low = csr.tril()
        lt = low.transpose()
        ga = gbo.Graph.from_csr(low, 32)
        gb = gbo.Graph.from_csr(lt, 32, gbo.FLAG_LAYOUT_COL)
        n = low.nrows
        drp = gbo.DeviceBuffer(8 * (n + 1))
        nnz = C.c_int64(0)
        gbo.check(gbo.lib().gbo_spgemm_nnz(ga.h, gb.h, drp.ptr, C.byref(nnz), None), "spgemm_nnz")
        m = int(nnz.value)
        dci, dv = gbo.DeviceBuffer(4 * max(m, 1)), gbo.DeviceBuffer(4 * max(m, 1))

        def run():
            gbo.check(gbo.lib().gbo_spgemm_nnz(ga.h, gb.h, drp.ptr, C.byref(nnz), None), "spgemm_nnz")
            gbo.check(gbo.lib().gbo_spgemm_fill(ga.h, gb.h, drp.ptr, dci.ptr, dv.ptr, None), "spgemm_fill")

        ms = _timed(gbo, run, max(1, args.steps // 2), args.warmup)
        total = ga.bmm_sum(gb)
        sum_ms = _timed(gbo, lambda: ga.bmm_sum(gb), args.steps, args.warmup)
        rp, ci, _ = ga.b2sr()
        brp, _, _ = gb.b2sr()
        pairs = int(np.diff(brp.astype(np.int64))[ci].sum())
        t0 = time.perf_counter()
        wrp, _, wv = oracle.spgemm_csr(low.rowptr, low.colind, n, lt.rowptr, lt.colind, lt.ncols)
        cpu_ms = (time.perf_counter() - t0) * 1e3
        res[name] = {"ms": ms, "nnz_c": m, "tile_pairs": pairs, "g_tile_pairs_per_s": pairs / (ms / 1e3) / 1e9,
                     "sum": total, "sum_ms": sum_ms, "matches_oracle": bool(int(wrp[-1]) == m and int(wv.sum()) == total),
                     "cpu_ms": cpu_ms, "cpu_threads": oracle.max_threads(), "vs_cpu": cpu_ms / ms,
                     "nnz_l": low.nnz}
        for x in (ga, gb):
            x.free()
    r = res["rmat14"]
    _line("ms", r["ms"], "ms per product (count + fill)", False, r["ms"], args,
          {"workload": "C = L L^T sparse output, R-MAT 14 ef16 seed 1 (lower triangle), B2SR 32 (L row words, "
                       "L^T column words)", "nnz_l": r["nnz_l"], "nnz_c": r["nnz_c"]},
          dtype="i32", by_graph=res,
          cpu_baseline={"value": r["cpu_ms"], "unit": "ms", "cores": r["cpu_threads"], "kind": "port",
                        "sample": "one oracle product (CSR Gustavson, bsrbmm/bsrbmm.cu:1273-1373 math)"})


def suite_ingest(args):
    """Matrix Market ingestion: R-MAT 20 (seed 0) written as a symmetric
    pattern .mtx (one triangle, 1-based), read by the host reader
    (gbo_read_mtx, readMtx semantics) and by the GPU reader
    (gbo_read_mtx_device), and packed by gbo_graph_from_mtx."""
    import tempfile

    import pandas as pd

    import gbo

    csr = gbo.gen_rmat(20, 16, seed=0, **RMAT)
    rows = np.repeat(np.arange(csr.nrows, dtype=np.int64), np.diff(csr.rowptr))
    keep = rows >= csr.colind
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "rmat20.mtx")
        with open(path, "w") as f:
            f.write("%%MatrixMarket matrix coordinate pattern symmetric\n")
            f.write(f"{csr.nrows} {csr.ncols} {int(keep.sum())}\n")
        pd.DataFrame({"i": rows[keep] + 1, "j": csr.colind[keep].astype(np.int64) + 1}).to_csv(
            path, sep=" ", header=False, index=False, mode="a")
        size = os.path.getsize(path)
        t0 = time.perf_counter()
        host = gbo.read_mtx(path)
        host_s = time.perf_counter() - t0
        dev = gbo.read_mtx_device(path)  # warm-up (and the check below)
        same = bool(np.array_equal(host.rowptr, dev.rowptr) and np.array_equal(host.colind, dev.colind))
        ts = []
        for _ in range(max(1, args.steps // 2)):
            t0 = time.perf_counter()
            gbo.read_mtx_device(path)
            ts.append(time.perf_counter() - t0)
        dev_s = float(np.median(ts))
        gs = []
        for _ in range(1 + max(1, args.steps // 2)):  # the first call is a warm-up
            t0 = time.perf_counter()
            g = gbo.Graph.from_mtx(path, gbo.MTX_READMTX, 0, 32, gbo.FLAG_SYMMETRIC)
            gbo.sync()
            gs.append(time.perf_counter() - t0)
            g.free()
        graph_s = float(np.median(gs[1:]))
    _line("GB/s", size / dev_s / 1e9, "GB/s of .mtx text parsed into a device CSR", True, dev_s * 1e3, args,
          {"workload": "R-MAT 20 ef16 seed 0, symmetric pattern .mtx (lower triangle), readMtx semantics",
           "file_bytes": size, "lines": int(keep.sum()), "nnz": host.nnz},
          dtype="u8", gpu_read_s=dev_s, host_read_s=host_s, speedup=host_s / dev_s, graph_from_mtx_s=graph_s,
          same_csr_as_host=same,
          cpu_baseline={"value": size / host_s / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
                        "sample": "one gbo_read_mtx of the same file (host parser, readMtx.hpp:351-423 semantics)"})


def suite_refgpu(args):
    """Reference arm, same-box GPU leg (--impl reference --workload refgpu).

    The reference's own kernels, compiled for sm_100a from its sources into
    oracle/_ref (oracle/Makefile), run on the same B200 beside this
    library's kernels on identical B2SR (packed by this library, byte-exact
    with the reference's csr2bsr_batch layout; the reference's packer is a
    host loop of cuSPARSE calls per block row and is not timed).  Graph: R-MAT
    scale 21 (seed 0), the largest R-MAT scale whose 32x32 B2SR stays inside
    the reference kernels' int32 word offsets (nblocks * 32 < 2^31).  Each
    pair is timed the way the reference's drivers time it (launches back to
    back between two events, bsrbmv/benchmark-bsrbmv.cu:1115-1126; the BFS
    loop of algorithm/bfs.cu:508-564 whole, with its per-level host copy)
    and compared output for output.  One JSON line per kernel pair."""
    import ctypes as C

    import gbo

    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    paths = [os.path.join(ref_dir, f) for f in ("librefbmv.so", "librefbmm.so")]
    if not all(os.path.exists(p) for p in paths):
        print(json.dumps({"impl": "reference", "workload": "refgpu",
                          "unavailable": "oracle/_ref not built (the reference checkout was absent at build time)"}),
              flush=True)
        return
    rb, rm = C.CDLL(paths[0]), C.CDLL(paths[1])
    P, I = C.c_void_p, C.c_int
    for nm in ("ref_bmv4_sparse", "ref_bmv8_sparse", "ref_bmv16_sparse_new", "ref_bmv32_sparse_new",
               "ref_bmv64_sparse_new"):
        getattr(rb, nm).argtypes = [P] * 5 + [I, I]
    rb.ref_bfs32_masked_v4.argtypes = [P, P, P, I, I, I, P, C.POINTER(C.c_float)]
    rb.ref_bmv32_sparse_full_minplus.argtypes = [P] * 5 + [I]
    rb.ref_bmv32_sparse_full.argtypes = [P] * 5 + [I, P, C.c_float]
    rm.ref_bmm32_sparse_masked_v5.argtypes = [P] * 7 + [I, I, I]
    gbo.check(gbo.lib().gbo_set_device(0), "set_device")
    e0, e1 = gbo.Event(), gbo.Event()
    steps, warm = max(3, args.steps), max(3, args.warmup)

    def timed(fn):
        for _ in range(warm):
            fn()
        gbo.sync()
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        gbo.sync()
        return e0.elapsed_ms(e1) / steps

    def chk(st, what):
        if st != 0:
            raise SystemExit(f"{what}: CUDA error {st}")

    def dev_b2sr(g):
        r, c, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
        gbo.check(gbo.lib().gbo_graph_b2sr(g.h, C.byref(r), C.byref(c), C.byref(v)), "graph_b2sr")
        return r.value, c.value, v.value

    def pad(a, m, fill):
        out = np.full(m, fill, dtype=a.dtype)
        out[:len(a)] = a
        return out

    def emit(kernel, ref_ms, our_ms, parity, config, **extra):
        line = {"impl": "reference", "workload": "refgpu", "metric": "ms", "unit": "ms per launch",
                "higher_is_better": False, "kernel_pair": kernel, "reference_ms": ref_ms, "ours_ms": our_ms,
                "speedup": ref_ms / our_ms, "steps": steps, "warmup": warm, "n_gpus": 1, "data": "synthetic",
                "parity": parity, "config": config}
        line.update(extra)
        print(json.dumps(line), flush=True)

    scale = args.ref_scale
    csr = gbo.gen_rmat(scale, EDGE_FACTOR, seed=SEED, **RMAT)
    n = csr.nrows
    cfg0 = {"graph": f"R-MAT scale {scale} ef16 seed {SEED} (a=0.57,b=0.19,c=0.19), symmetrised, deduplicated",
            "nvertices": n, "nnz": csr.nnz, "l2": "inputs larger than L2 (B2SR far above 126 MB)"}
    x01 = (np.random.default_rng(0).random(n) < 0.5).astype(np.int32)

    # --- BMV count at every tile width: bmv{4,8}_sparse, bmv{16,32,64}_sparse_new
    ref_names = {4: "ref_bmv4_sparse", 8: "ref_bmv8_sparse", 16: "ref_bmv16_sparse_new",
                 32: "ref_bmv32_sparse_new", 64: "ref_bmv64_sparse_new"}
    ref_src = {4: "algorithm/bsrbmv.cu:262", 8: "algorithm/bsrbmv.cu:310",
               16: "algorithm/bsrbmv.cu:2776", 32: "algorithm/bsrbmv.cu:2937", 64: "algorithm/bsrbmv.cu:3046"}
    peak, psrc = load_peaks()
    for b in [int(t) for t in args.ref_widths.split(",")]:
        g = gbo.Graph.from_csr(csr, b, gbo.FLAG_SYMMETRIC)
        inf = g.info()
        nblk, nbr = int(inf.nblocks), inf.nblockrows
        if nblk * b >= 2 ** 31:
            print(json.dumps({"impl": "reference", "workload": "refgpu", "kernel_pair": f"bmv count b={b}",
                              "skipped": f"{nblk} tiles: past the reference kernels' int32 word offsets"}))
            g.free()
            continue
        r, c, v = dev_b2sr(g)
        dx = gbo.DeviceBuffer.from_numpy(pad(gbo.bits_from_numpy(x01, b), inf.nblockcols + 64, 0))
        dref = gbo.DeviceBuffer.zeros(4 * (nbr + 64) * b)
        fn = getattr(rb, ref_names[b])
        run_ref = lambda: fn(v, dx.ptr, dref.ptr, r, c, nbr, nblk)
        chk(run_ref(), ref_names[b])
        gbo.sync()
        ref_y = dref.to_numpy(np.float32, n).astype(np.int64)
        dy = gbo.DeviceBuffer(4 * n)
        g.bmv_count(dx, dy)
        ours = dy.to_numpy(np.int32, n).astype(np.int64)
        keep = np.ones(n, bool)
        note = None
        if b == 64:
            # bmv64_sparse_new packs rows r and r+32 as 16-bit halves of one
            # word (bsrbmv.cu:3084-3090): rows whose pair holds a count past
            # 32767 overflow there and are left out of the comparison
            big = np.zeros((nbr * 64,), bool)
            big[:n] = ours > 32767
            pair = big.reshape(nbr, 2, 32).any(axis=1)
            keep = np.repeat(pair[:, None, :], 2, axis=1).reshape(-1)[:n] == False  # noqa: E712
            note = f"{int((~keep).sum())} rows beside a count > 32767 excluded (reference 16-bit halves)"
        mism = int(np.count_nonzero(ours[keep] != ref_y[keep]))
        t_ref = timed(run_ref)
        t_ours = timed(lambda: g.bmv_count(dx, dy))
        by = _bmv_bytes(inf, b, n, max(1, b // 8) * inf.nblockcols + 4 * n)
        emit(f"BMV count b={b}: {ref_names[b][4:]} ({ref_src[b]}) vs gbo_bmv_count", t_ref, t_ours,
             {"checked": f"int32 row counts of all {n} rows", "mismatched_rows": mism, "equal": mism == 0,
              **({"note": note} if note else {})},
             dict(cfg0, tile_bits=b, nblocks=nblk),
             algorithmic_bytes=by, ours_gbs=by / (t_ours / 1e3) / 1e9, ref_gbs=by / (t_ref / 1e3) / 1e9,
             ours_frac=by / (t_ours / 1e3) / 1e9 / peak, ref_frac=by / (t_ref / 1e3) / 1e9 / peak,
             peak_gbs=peak, peak_source=psrc)
        for buf in (dx, dref, dy):
            buf.free()
        g.free()

    # --- 32x32 graph for the BFS loop, min-plus, fp32
    g = gbo.Graph.from_csr(csr, 32, gbo.FLAG_SYMMETRIC)
    inf = g.info()
    nblk, nbr = int(inf.nblocks), inf.nblockrows
    r, c, v = dev_b2sr(g)
    cfg = dict(cfg0, tile_bits=32, nblocks=nblk)

    succ = np.zeros(64, np.int32)
    ms = C.c_float(0)
    it = rb.ref_bfs32_masked_v4(v, r, c, nbr, 0, 64, succ.ctypes.data, C.byref(ms))
    if it < 0:
        raise SystemExit("reference BFS loop: CUDA error")
    ref_times = []
    for _ in range(steps):
        rb.ref_bfs32_masked_v4(v, r, c, nbr, 0, 64, succ.ctypes.data, C.byref(ms))
        ref_times.append(ms.value)
    lv, depth = g.bfs(0)
    d_lv = gbo.DeviceBuffer(4 * n)
    t_ours = timed(lambda: g.bfs(0, out=d_lv))
    hist = np.bincount(lv[lv > 0], minlength=it + 1)[1:it + 1]
    edges = traversed_edges(csr, lv)
    t_ref = float(np.median(ref_times))
    emit("BFS from vertex 0: the bfs.cu:508-564 loop (bmv32_sparse_bin_masked_v4, bsrbmv.cu:740) vs gbo_bfs",
         t_ref, t_ours,
         {"checked": "vertices reached per level (the reference loop's succ sequence) against gbo_bfs's level "
                     "histogram", "reference_succ": succ[:it].tolist(), "equal": bool(np.array_equal(hist, succ[:it]))},
         cfg, ref_gteps=edges / (t_ref / 1e3) / 1e9, ours_gteps=edges / (t_ours / 1e3) / 1e9,
         reference_iterations=int(it), ours_depth=int(depth))
    d_lv.free()

    npad = nbr * 32
    rng = np.random.default_rng(8)
    # min-plus (sssp.cu:447)
    d = rng.integers(0, 40, n).astype(np.uint32)
    d[rng.random(n) < 0.3] = np.uint32(2147483647)
    dd = gbo.DeviceBuffer.from_numpy(pad(d, npad, np.uint32(2147483647)))
    dref = gbo.DeviceBuffer.zeros(4 * npad)
    run_ref = lambda: rb.ref_bmv32_sparse_full_minplus(v, dd.ptr, dref.ptr, r, c, nbr)
    chk(run_ref(), "minplus")
    gbo.sync()
    dy = gbo.DeviceBuffer(4 * n)
    g.bmv_minplus(dd, dy)
    rp, ci, _ = g.b2sr()
    row_of = np.repeat(np.arange(nbr), np.diff(rp))
    diag = np.zeros(nbr, bool)
    diag[row_of[ci == row_of]] = True
    rows = np.repeat(diag, 32)[:n]
    mism = int(np.count_nonzero(dy.to_numpy(np.uint32, n)[rows] != dref.to_numpy(np.uint32, n)[rows]))
    t_ref, t_ours = timed(run_ref), timed(lambda: g.bmv_minplus(dd, dy))
    emit("min-plus BMV: bmv32_sparse_full_minplus (bsrbmv.cu:1083, sssp.cu:447) vs gbo_bmv_minplus", t_ref, t_ours,
         {"checked": f"uint32 results of the {int(rows.sum())} rows whose block row stores its diagonal tile "
                     "(the reference adds the 0-weight diagonal only there)", "mismatched_rows": mism,
          "equal": mism == 0}, cfg)
    for bf in (dd, dref, dy):
        bf.free()

    # fp32 PageRank BMV (pr.cu:482): y = alpha * sum p[j] / outdeg(j)
    p = rng.random(n).astype(np.float32)
    dp = gbo.DeviceBuffer.from_numpy(pad(p, npad, np.float32(0)))
    drp = gbo.DeviceBuffer.from_numpy(pad(csr.rowptr, npad + 1, csr.rowptr[-1]))
    dref = gbo.DeviceBuffer.zeros(4 * npad)
    run_ref = lambda: rb.ref_bmv32_sparse_full(v, dp.ptr, dref.ptr, r, c, nbr, drp.ptr, 0.85)
    chk(run_ref(), "full")
    gbo.sync()
    dy = gbo.DeviceBuffer(4 * n)
    run_ours = lambda: gbo.check(gbo.lib().gbo_bmv_float_degptr(g.h, dp.ptr, dy.ptr, C.c_float(0.85), drp.ptr,
                                                                 None), "bmv_float_degptr")
    run_ours()
    a64 = dy.to_numpy(np.float32, n).astype(np.float64)
    b64 = dref.to_numpy(np.float32, n).astype(np.float64)
    rel = float(np.abs(a64 - b64).sum() / max(np.abs(b64).sum(), 1e-300))
    t_ref, t_ours = timed(run_ref), timed(run_ours)
    it_c = C.c_int(0)
    dpr = gbo.DeviceBuffer(4 * n)
    gbo.check(gbo.lib().gbo_pagerank(g.h, C.c_float(0.85), 20, C.c_float(-1.0), dpr.ptr, C.byref(it_c), None), "pr")
    pr_step = float(np.mean(g.last_run()["step_ms"]))
    emit("fp32 BMV: bmv32_sparse_full (bsrbmv.cu:1239, pr.cu:482) vs gbo_bmv_float_degptr", t_ref, t_ours,
         {"checked": f"fp32 y of all {n} rows, relative L1 (reference sums in fp32, this library in fp64)",
          "rel_l1": rel, "equal": bool(rel <= 1e-5)}, cfg, ours_pagerank_iteration_ms=pr_step)
    for bf in (dp, drp, dref, dy, dpr):
        bf.free()
    g.free()

    # --- masked BMM / triangle counting (bsrbmm.cu:1214, tc.cu:948)
    tcg = {"mesh": ("king mesh 4096x4096", lambda: gbo.gen_king_mesh(4096)),
           "rmat": ("R-MAT scale 20 ef16 seed 1", lambda: gbo.gen_rmat(20, 16, seed=1, **RMAT))}
    for key in args.tc_graphs.split(","):
        name, make = tcg[key]
        tcsr = make()
        low = tcsr.tril()
        ga = gbo.Graph.from_csr(low, 32)
        gb = gbo.Graph.from_csr(low.transpose(), 32, gbo.FLAG_LAYOUT_COL)
        ar, ac, av = dev_b2sr(ga)
        br, bc, bv = dev_b2sr(gb)
        ia = ga.info()
        dcount = gbo.DeviceBuffer.zeros(4)
        run_ref = lambda: rm.ref_bmm32_sparse_masked_v5(av, bv, dcount.ptr, ar, ac, br, bc, ia.nblockrows,
                                                        int(ia.nblocks), tcsr.nrows)
        e0.record()
        chk(run_ref(), "masked_v5")
        e1.record()
        gbo.sync()
        t_once = e0.elapsed_ms(e1)
        ref_tri = int(dcount.to_numpy(np.int32, 1)[0])
        gl = gbo.Graph.from_csr(tcsr, 32, gbo.FLAG_LOWER)
        ours = gl.tc()
        # a reference launch of more than a second is timed once (R-MAT 20:
        # its per-tile search is quadratic in the hub block rows)
        t_ref = timed(run_ref) if t_once < 1000.0 else t_once
        t_ours = timed(gl.tc)
        gd = gbo.Graph.from_csr(tcsr, 16 if key == "mesh" else 8, gbo.FLAG_LOWER | gbo.FLAG_DEGREE_ORDER)
        t_best = timed(gd.tc)
        emit(f"triangle count, {name}: bmm32_sparse_masked_v5 (bsrbmm.cu:1214) vs gbo_tc (b = 32, input order)",
             t_ref, t_ours, {"checked": "triangle count", "reference": ref_tri, "ours": ours,
                             "equal": ref_tri == ours},
             {"graph": name, "nvertices": tcsr.nrows, "nnz": tcsr.nnz, "tile_bits": 32,
              "nblocks_L": int(ia.nblocks)},
             ours_degree_order_ms=t_best, ours_degree_order_tile=16 if key == "mesh" else 8,
             speedup_degree_order=t_ref / t_best)
        for x in (ga, gb, gl, gd):
            x.free()


def suite_noalloc(args):
    """BMV count straight from caller-owned B2SR arrays (gbo_bmv_count_noalloc,
    no allocation) against the graph-handle BMV (gbo_bmv_count) on R-MAT 14,
    17 and 20 at b = 32, x of density 0.5: time per call and equal counts."""
    import gbo

    peak, psrc = load_peaks()
    rows = {}
    for scale in (14, 17, 20):
        csr = gbo.gen_rmat(scale, EDGE_FACTOR, seed=SEED, **RMAT)
        g = gbo.Graph.from_csr(csr, 32)
        rp, ci, w = g.b2sr()
        n = csr.nrows
        drp, dci, dv = (gbo.DeviceBuffer.from_numpy(a) for a in (rp, ci, w))
        x = (np.random.default_rng(0).random(n) < 0.5).astype(np.int32)
        dx = gbo.DeviceBuffer.from_numpy(gbo.bits_from_numpy(x, 32))
        y1, y2 = gbo.DeviceBuffer(4 * n), gbo.DeviceBuffer(4 * n)
        handle_ms = _timed(gbo, lambda: g.bmv_count(dx, y1), 20, args.warmup)
        na_ms = _timed(gbo, lambda: gbo.check(gbo.lib().gbo_bmv_count_noalloc(
            n, n, 32, len(ci), drp.ptr, dci.ptr, dv.ptr, dx.ptr, y2.ptr, gbo.OUT_I32, 0, None), "bmv_noalloc"),
            20, args.warmup)
        # the BMV model: tiles (128-byte words + 4-byte column), block-row
        # offsets, x words (one per block column) and y
        by = len(ci) * (32 * 32 // 8 + 4) + 4 * len(rp) + 4 * (len(rp) - 1) + 4 * n
        rows[f"rmat{scale}"] = {"tiles": int(len(ci)), "noalloc_ms": na_ms, "handle_ms": handle_ms,
                                "noalloc_frac": by / (na_ms / 1e3) / 1e9 / peak,
                                "equal": bool(np.array_equal(y1.to_numpy(np.int32, n), y2.to_numpy(np.int32, n)))}
        g.free()
    top = rows["rmat20"]
    _line("ms", top["noalloc_ms"], "ms per call", False, top["noalloc_ms"], args,
          {"workload": "gbo_bmv_count_noalloc vs gbo_bmv_count, R-MAT 14/17/20 (seed 0), B2SR 32, x density 0.5"},
          dtype="u32", by_graph=rows, peak_source=psrc,
          parity={"checked": "int32 counts of the two entry points, every row", "equal": all(r["equal"] for r in rows.values())})


SUITE = {
    "sssp": lambda a: suite_config2(a, "sssp"),
    "cc": lambda a: suite_config2(a, "cc"),
    "pr": lambda a: suite_config2(a, "pr"),
    "tc": suite_tc,
    "msbfs": suite_msbfs,
    "batch": suite_batch,
    "ppr": suite_ppr,
    "serve": suite_serve,
    "spgemm": suite_spgemm,
    "ingest": suite_ingest,
    "noalloc": suite_noalloc,
}


def main():
    args = parse()
    _Nvtx.on = args.nvtx
    ws, rank, local = dist_env()
    if args.impl == "reference":
        if args.workload == "refgpu":
            if rank == 0:
                suite_refgpu(args)
        else:
            run_reference(args, ws, rank)
        return
    if args.workload == "refgpu":
        raise SystemExit("--workload refgpu belongs to the reference arm: add --impl reference")
    if args.workload != "bfs":
        import gbo

        gbo.check(gbo.lib().gbo_set_device(local), "set_device")
        if rank == 0:
            SUITE[args.workload](args)
        return
    run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
