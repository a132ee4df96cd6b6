"""Generates tests/golden/golden.json: known answers for the parity tests.

Answers come from independent third-party code (networkx, scipy), never from
the oracle or libgbo's kernels, so they pin the oracle.  Inputs are
(1) the reference's own fixture files, read in place from the reference
checkout when it is present (bsrbmv/test.mtx, bsrbmm/test.mtx, G43.mtx --
only derived answers are stored, never the matrices), and (2) graphs from
libgbo's seeded host generators (ER n=1000 p=0.02002 seed 0, R-MAT scale 12,
king meshes), whose CSR is regenerated at test time.

Run:  python tests/golden/make_golden.py [reference_root]
"""
import hashlib
import json
import os
import sys

import networkx as nx
import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "graph-bit-ops_b200"))
import gbo  # noqa: E402  (host-side reader/generators only)

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GBO_REF_DIR", "/root/reference")


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def answers(csr, x_seed=0, src=0):
    n = csr.nrows
    A = sp.csr_matrix((np.ones(csr.nnz, np.int64), csr.colind, csr.rowptr), shape=(n, csr.ncols))
    rng = np.random.default_rng(x_seed)
    x = (rng.random(csr.ncols) < 0.5).astype(np.int64)
    y = A @ x  # counts with duplicates; fixtures here are duplicate-free
    G = nx.DiGraph()
    G.add_nodes_from(range(n))
    r, c = A.nonzero()
    # P pulls x[j] into row i, so BFS follows edges j -> i
    G.add_edges_from(zip(c.tolist(), r.tolist()))
    lv = np.full(n, -1, np.int64)
    for v, d in nx.single_source_shortest_path_length(G, src).items():
        lv[v] = d
    out = {
        "n": n, "nnz": int(csr.nnz), "rowptr_sha": sha(csr.rowptr), "colind_sha": sha(csr.colind),
        "bmv_x_seed": x_seed, "bmv_count_sha": sha(y.astype(np.int32)), "bmv_count_sum": int(y.sum()),
        "bfs_src": src, "bfs_levels_sha": sha(lv.astype(np.int32)),
        "bfs_depth": int(lv.max() + 1), "bfs_reached": int((lv >= 0).sum()),
    }
    sym = (A != A.T).nnz == 0
    if sym:
        U = nx.Graph()
        U.add_nodes_from(range(n))
        U.add_edges_from((i, j) for i, j in zip(r.tolist(), c.tolist()) if i != j)
        out["triangles"] = int(sum(nx.triangles(U).values()) // 3)
        comps = list(nx.connected_components(U))
        lab = np.zeros(n, np.int64)
        for cpt in comps:
            lab[list(cpt)] = min(cpt)
        out["components"] = len(comps)
        out["cc_labels_sha"] = sha(lab.astype(np.int32))
    # PageRank of the reference's recurrence (pr.cu:449-513) in fp64 with scipy:
    # p' = alpha * P D^-1 p + (1-alpha)/n, D = column counts of P, 20 iterations
    deg = np.asarray(A.sum(axis=0)).ravel().astype(np.float64)
    inv = np.divide(1.0, deg, out=np.zeros_like(deg), where=deg > 0)
    p = np.full(n, 1.0 / n)
    for _ in range(20):
        p = 0.85 * (A @ (p * inv)) + 0.15 / n
    out["pr20"] = [float(v) for v in p[:8]]
    out["pr20_sum"] = float(p.sum())
    return out


def main():
    g = {}
    fixtures = {
        "bsrbmv_test": "bsrbmv/test.mtx",
        "bsrbmm_test": "bsrbmm/test.mtx",
        "G43": "bsrbmv/G43.mtx",
    }
    for key, rel in fixtures.items():
        path = os.path.join(REF, rel)
        if not os.path.exists(path):
            continue
        for mode, mname in ((gbo.MTX_READMTX, "readmtx"), (gbo.MTX_MMIO, "mmio")):
            csr = gbo.read_mtx(path, mode, 0)
            g[f"{key}_{mname}"] = answers(csr)
    g["er1000"] = answers(gbo.gen_er(1000, 0.02002, 0))
    g["rmat12"] = answers(gbo.gen_rmat(12, 16, seed=0))
    for side in (2, 3, 8, 33):
        m = gbo.gen_king_mesh(side)
        a = answers(m)
        a["triangles_closed_form"] = 4 * (side - 1) ** 2
        a["edges_closed_form"] = 2 * side * (side - 1) + 2 * (side - 1) ** 2
        g[f"mesh{side}"] = a
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(g, f, indent=1, sort_keys=True)
    print("wrote", len(g), "entries")


if __name__ == "__main__":
    main()
