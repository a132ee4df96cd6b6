"""The reference-style C++ driver built on include/gbo_compat.hpp (the drop-in
path for the reference's drivers) against the oracle."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
DRIVER = os.path.join(ROOT, "graph-bit-ops_b200", "examples", "bfs_driver")


def write_mtx(path, csr, symmetric):
    rows = np.repeat(np.arange(csr.nrows), np.diff(csr.rowptr))
    cols = csr.colind
    if symmetric:
        keep = rows >= cols
        rows, cols = rows[keep], cols[keep]
    kind = "symmetric" if symmetric else "general"
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate pattern {kind}\n")
        f.write(f"{csr.nrows} {csr.ncols} {len(rows)}\n")
        for r, c in zip(rows.tolist(), cols.tolist()):
            f.write(f"{r + 1} {c + 1}\n")


@pytest.mark.parametrize("which", ["er1000", "rmat12", "directed"])
def test_compat_driver(gbo, orc, gpu, tmp_path, which):
    assert os.path.exists(DRIVER), "build the example with make in graph-bit-ops_b200"
    if which == "er1000":
        csr, sym = gbo.gen_er(1000, 0.02002, 0), True
    elif which == "rmat12":
        csr, sym = gbo.gen_rmat(12, 16, seed=0), True
    else:
        rng = np.random.default_rng(3)
        csr = gbo.csr_from_edges(rng.integers(0, 900, 5000), rng.integers(0, 900, 5000), 900, False, True)
        sym = False
    p = tmp_path / "g.mtx"
    write_mtx(str(p), csr, sym)
    out = subprocess.run([DRIVER, str(p), "0"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.splitlines()
    succ = [int(l.split(":")[1]) for l in lines if l.startswith("succ:")]
    # BFS from 0 along A's edges: P = A^T
    at = csr.transpose()
    lv, depth = orc.bfs_csr(at.rowptr, at.colind, at.nrows, 0)
    hist = [int((lv == L + 1).sum()) for L in range(depth)]
    assert succ == hist
    dline = [l for l in lines if l.startswith("gbo_bfs depth:")][0].split()
    assert int(dline[2]) == depth and int(dline[4]) == int((lv >= 0).sum())
    if sym:
        tline = [l for l in lines if l.startswith("ntris:")][0].split()
        assert int(tline[1]) == orc.tc_csr(csr.rowptr, csr.colind, csr.nrows)
