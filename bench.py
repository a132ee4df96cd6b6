"""Benchmark: BFS GTEPS on B2SR (bit-packed BSR) on B200, plus the roofline of
the BFS pull kernel, the plain BSR-BMV roofline and a CPU baseline.

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
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving streams")
    ap.add_argument("--serve-qps", type=float, default=4000.0, help="offered BFS query rate")
    ap.add_argument("--serve-s", type=float, default=1.5, help="seconds of arrivals per stream")
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
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
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


def workload_name(scale, tile):
    return (f"BFS from vertex 0, R-MAT scale {scale} edge factor {EDGE_FACTOR} "
            f"(a=0.57,b=0.19,c=0.19, seed {SEED}, symmetrised, deduplicated), B2SR {tile}x{tile}")


def traversed_edges(csr, levels):
    deg = np.diff(csr.rowptr).astype(np.int64)
    return int(deg[levels >= 0].sum() // 2)


# --------------------------------------------------------------- roofline
def bfs_level_bytes(rowptr_b, colind_b, levels, nrows, b):
    """Algorithmic bytes of each BFS pull step (the words the step must touch).

    Step L reads the block-row offsets, the visited and frontier words, the
    block-column index of every tile in a block row that still has an
    unvisited vertex, and -- only for tiles whose frontier segment is non-empty
    -- one b-bit row word per unvisited row; it writes the next frontier
    words, visited words of changed rows and one int32 level per new vertex.
    """
    nbr = len(rowptr_b) - 1
    wb = max(1, b // 8)
    pad = np.full(nbr * b, -2, np.int64)
    pad[:nrows] = levels
    lv = pad.reshape(nbr, b)
    depth = int(levels.max()) + 1
    row_of = np.repeat(np.arange(nbr, dtype=np.int64), np.diff(rowptr_b))
    out = []
    for L in range(depth):
        visited = (lv >= 0) & (lv <= L)
        unvis = ((lv == -1) | (lv > L)).sum(axis=1)  # real unvisited rows
        front_nz = (lv == L).any(axis=1)
        open_row = unvis > 0
        t_open = open_row[row_of]
        t_need = t_open & front_nz[colind_b]
        newv = int((lv == L + 1).sum())
        changed = int(((lv == L + 1).any(axis=1)).sum())
        by = 4 * (nbr + 1) + 2 * wb * nbr + wb * changed + 4 * newv
        by += 4 * int(t_open.sum())
        by += wb * int(unvis[row_of[t_need]].sum())
        out.append(by)
        del visited
    return out


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(name):
    """Per-launch DRAM bytes of a kernel from a committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.startswith("traffic_bytes_per_launch:"):
                try:
                    return float(line.split(":", 1)[1])
                except ValueError:
                    return None
    return None


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
def cpu_bfs(csr, tile, samples):
    """The oracle's port of the reference BFS loop (algorithm/bfs.cu:508-564)
    on B2SR with OpenMP over block rows; returns (GTEPS, seconds, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    bs = oracle.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, tile)
    lv, _ = oracle.bfs_b2sr(bs, 0)
    edges = traversed_edges(csr, lv)
    times = []
    for _ in range(max(1, samples)):
        t0 = time.perf_counter()
        oracle.bfs_b2sr(bs, 0)
        times.append(time.perf_counter() - t0)
    t = float(np.median(times))
    return edges / t / 1e9, t, oracle.max_threads(), edges


def run_reference(args, ws, rank):
    """--impl reference: the reference path's CPU restatement (the reference
    has no CPU implementation of its own; its drivers need a GPU and removed
    cuSPARSE APIs), all host threads, same workload, metric and unit."""
    if rank != 0:
        return
    import gbo

    csr = gbo.gen_rmat(args.scale, EDGE_FACTOR, seed=SEED, **RMAT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    bs = oracle.pack(csr.rowptr, csr.colind, csr.nrows, csr.ncols, args.tile)
    lv, _ = oracle.bfs_b2sr(bs, 0)
    edges = traversed_edges(csr, lv)
    for _ in range(args.warmup):
        oracle.bfs_b2sr(bs, 0)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.bfs_b2sr(bs, 0)
    dt = (time.perf_counter() - t0) / args.steps
    v = edges / dt / 1e9
    line = {
        "impl": "reference", "metric": "GTEPS", "value": v, "unit": "GTEPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": workload_name(args.scale, args.tile), "scale": args.scale,
                   "tile_bits": args.tile, "traversed_edges": edges},
        "cpu_baseline": {"value": v, "unit": "GTEPS", "cores": oracle.max_threads(), "kind": "port",
                         "sample": f"{args.steps} full BFS runs from vertex 0 (oracle port of "
                                   "algorithm/bfs.cu:508-564 on B2SR, OpenMP over block rows)"},
        "e2e": {"value": v, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- serving
def serve_stream(gbo, g, n, rate_qps, duration_s, ppr_frac, seed):
    """Poisson arrivals of BFS sources and PPR sets (1..64 vertices, Dirichlet
    weights) into the continuous-batching server; returns achieved qps and
    p50/p99 latencies (submit to result in host memory)."""
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
    srv = gbo.Server(g, bfs_slots=1024, ppr_slots=32 if ppr_frac > 0 else 0, alpha=0.85, tol=1e-7)
    import queue

    tq = queue.Queue()
    lat = {"bfs": [], "ppr": []}
    lock = threading.Lock()
    t0 = time.perf_counter()

    def producer():
        t = t0
        for i in range(nq):
            t += gaps[i]
            d = t - time.perf_counter()
            if d > 0:
                time.sleep(d)
            kind, arg = qs[i]
            tq.put((kind, srv.submit_bfs(arg) if kind == "bfs" else srv.submit_ppr(*arg)))
        for _ in range(consumers):
            tq.put(None)

    def consumer():
        while True:
            item = tq.get()
            if item is None:
                return
            kind, ticket = item
            _, ms, _ = srv.wait(ticket, kind, timeout=600.0)
            with lock:
                lat[kind].append(ms)

    consumers = 8
    ths = [threading.Thread(target=producer)] + [threading.Thread(target=consumer) for _ in range(consumers)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    out = {"offered_qps": rate_qps, "queries": nq, "achieved_qps": nq / wall, "wall_s": wall,
           "rounds": st["rounds"]}
    for k, v in lat.items():
        if v:
            out[f"{k}_p50_ms"] = float(np.percentile(v, 50))
            out[f"{k}_p99_ms"] = float(np.percentile(v, 99))
            out[f"{k}_count"] = len(v)
    return out


# ------------------------------------------------------------- our arm
def run_ours(args, ws, rank, local):
    import gbo

    gbo.check(gbo.lib().gbo_set_device(local), "set_device")
    dist = Dist(ws)
    csr = gbo.gen_rmat(args.scale, EDGE_FACTOR, seed=SEED, **RMAT)
    t0 = time.perf_counter()
    g = gbo.Graph.from_csr(csr, args.tile)
    build_s = time.perf_counter() - t0
    info = g.info()
    n = csr.nrows
    d_level = gbo.DeviceBuffer(4 * n)

    # correctness of the timed path against an independent CPU BFS (rank 0)
    levels, depth = g.bfs(0)
    edges = traversed_edges(csr, levels)

    clocks = ClockSampler(local)  # samples from the warm-up to the end of the timed runs
    for _ in range(args.warmup):
        g.bfs(0, out=d_level)
    ev0, ev1 = gbo.Event(), gbo.Event()
    step_ms_all, launches = [], 0
    dist.barrier()
    gbo.sync()
    ev0.record()
    for _ in range(args.steps):
        g.bfs(0, out=d_level)
        st = g.last_run()
        step_ms_all.extend(st["step_ms"])
        launches += st["kernel_launches"]
    ev1.record()
    gbo.sync()
    dist.barrier()
    ms = ev0.elapsed_ms(ev1) / args.steps
    ms_max = dist.max(ms)

    # e2e: same call with the result read back into pinned host memory
    h_level = C_pinned(4 * n)
    for _ in range(1):
        g.bfs(0, out=d_level)
    dist.barrier()
    gbo.sync()
    ev0.record()
    for _ in range(args.steps):
        g.bfs(0, out=d_level)
        gbo.check(gbo.lib().gbo_memcpy_d2h(h_level.ptr, d_level.ptr, 4 * n, None), "d2h")
    ev1.record()
    gbo.sync()
    dist.barrier()
    e2e_ms = dist.max(ev0.elapsed_ms(ev1) / args.steps)

    # roofline of the BFS pull kernel: algorithmic bytes per level / its
    # event-timed duration inside the timed runs
    rp, ci, _ = None, None, None
    r = C_void()
    c = C_void()
    gbo.check(gbo.lib().gbo_graph_b2sr(g.h, r.ref(), c.ref(), None), "graph_b2sr")
    rowptr_b = gbo.device_to_numpy(r.value, np.int32, info.nblockrows + 1)
    colind_b = gbo.device_to_numpy(c.value, np.int32, int(info.nblocks))
    lvl_bytes = bfs_level_bytes(rowptr_b, colind_b, levels, n, args.tile)
    per_level_ms = np.array(step_ms_all, np.float64).reshape(args.steps, -1)
    lvl_ms = per_level_ms.mean(axis=0)
    k = min(len(lvl_bytes), len(lvl_ms))
    peak, peak_src = load_peaks()
    achieved = sum(lvl_bytes[:k]) / (sum(lvl_ms[:k]) / 1e3) / 1e9
    traffic = load_traffic("bfs_step_rmat22_b32.md")

    # plain BSR-BMV count roofline on the same graph (random x, density 0.5)
    x = (np.random.default_rng(0).random(n) < 0.5).astype(np.int32)
    xw = gbo.bits_from_numpy(x, args.tile)
    dx = gbo.DeviceBuffer.from_numpy(xw)
    dy = gbo.DeviceBuffer(4 * n)
    for _ in range(3):
        g.bmv_count(dx, dy)
    gbo.sync()
    ev0.record()
    nb = 20
    for _ in range(nb):
        g.bmv_count(dx, dy)
    ev1.record()
    gbo.sync()
    bmv_ms = ev0.elapsed_ms(ev1) / nb
    clk = clocks.stop()

    # batched: k sources per multi-source BFS (bit frontier matrix) vs one
    # source per plain BFS, same graph, queries per second
    batched = {}
    rng = np.random.default_rng(3)
    for kq in (64, 1024):
        srcs = rng.integers(0, n, kq).astype(np.int32)
        d_lv = gbo.DeviceBuffer(4 * n * kq)
        g.msbfs(srcs, out=d_lv)
        gbo.sync()
        reps = 3
        ev0.record()
        for _ in range(reps):
            g.msbfs(srcs, out=d_lv)
        ev1.record()
        gbo.sync()
        mms = ev0.elapsed_ms(ev1) / reps
        batched[f"k{kq}"] = {"ms": mms, "qps": kq / (mms / 1e3),
                            "qps_vs_plain": (kq / mms) / (1.0 / ms)}
        d_lv.free()

    # served: Poisson query streams into the continuous-batching server
    served = {}
    if not args.no_serve:
        served["bfs_only"] = serve_stream(gbo, g, n, args.serve_qps, args.serve_s, 0.0, 5)
        served["bfs_only"]["vs_plain_bfs_qps"] = served["bfs_only"]["achieved_qps"] / (1e3 / ms)
        served["mixed_10pct_ppr"] = serve_stream(gbo, g, n, args.serve_qps / 8, args.serve_s, 0.1, 6)
    wb = max(1, args.tile // 8)
    bmv_bytes = (int(info.nblocks) * (args.tile * args.tile // 8 + 4) + 4 * (info.nblockrows + 1)
                 + wb * info.nblockcols + 4 * n)
    bmv_gbs = bmv_bytes / (bmv_ms / 1e3) / 1e9

    gteps = ws * edges / (ms_max / 1e3) / 1e9
    line = {
        "metric": "GTEPS", "value": gteps, "unit": "GTEPS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": workload_name(args.scale, args.tile), "scale": args.scale,
                   "tile_bits": args.tile, "nvertices": n, "nnz": csr.nnz,
                   "nblocks": int(info.nblocks), "b2sr_gb": info.b2sr_bytes / 1e9,
                   "traversed_edges": edges, "bfs_depth": depth,
                   "l2": "inputs larger than L2 (B2SR tiles far above 126 MB)",
                   "parallelism": "replicas" if ws > 1 else "single"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": f"k_bfs_step<{args.tile}> (BFS pull step, mean over levels)",
                     "peak_source": peak_src,
                     "algorithmic_bytes_per_launch": float(np.mean(lvl_bytes[:k])),
                     "ms_per_launch": float(np.mean(lvl_ms[:k]))},
        "e2e": {"value": ws * edges / (e2e_ms / 1e3) / 1e9, "unit": "GTEPS",
                "h2d_bytes_per_step": 4, "d2h_bytes_per_step": 4 * n},
        "gpu_launches": int(launches),
        "clocks": clk,
        "bmv_count": {"achieved_gbs": bmv_gbs, "frac": bmv_gbs / peak, "ms": bmv_ms,
                      "algorithmic_bytes": bmv_bytes, "gteps": csr.nnz / (bmv_ms / 1e3) / 1e9},
        "batched_bfs": dict(batched, plain_qps=1e3 / ms),
        "served": served,
        "levels_ms": [float(v) for v in lvl_ms[:k]],
        "levels_gb": [b / 1e9 for b in lvl_bytes[:k]],
        "graph_build_s": build_s,
    }
    if rank == 0 and ws == 1 and not args.no_cpu:
        v, t, cores, _ = cpu_bfs(csr, args.tile, args.cpu_samples)
        line["cpu_baseline"] = {"value": v, "unit": "GTEPS", "cores": cores, "kind": "port",
                                "sample": f"{args.cpu_samples} full BFS runs from vertex 0 "
                                          f"(median {t:.2f} s), oracle port of algorithm/bfs.cu:508-564"}
    if rank == 0:
        print(json.dumps(line), flush=True)
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


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
