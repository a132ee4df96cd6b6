"""Seeded input graphs shared by the GPU parity tests."""
import numpy as np


def star(gbo, n):
    """Vertex 0 joined to all others: block row 0 has every block column, so it
    is split across warps at every tile width."""
    src = np.zeros(n - 1, np.int32)
    dst = np.arange(1, n, dtype=np.int32)
    return gbo.csr_from_edges(src, dst, n, True, True)


def ragged(gbo, n=1001, seed=4):
    """Random directed graph with empty rows and a row count that is not a
    multiple of any tile width."""
    rng = np.random.default_rng(seed)
    src = rng.integers(0, n // 2, 6 * n)  # rows >= n/2 stay empty
    dst = rng.integers(0, n, 6 * n)
    return gbo.csr_from_edges(src, dst, n, False, True)


def cases(gbo):
    return {
        "er1000": gbo.gen_er(1000, 0.02002, 0),
        "rmat12": gbo.gen_rmat(12, 16, seed=0),
        "rmat14": gbo.gen_rmat(14, 8, seed=2),
        "mesh33": gbo.gen_king_mesh(33),
        "star20000": star(gbo, 20000),
        "ragged1001": ragged(gbo),
        "single": gbo.csr_from_edges([0], [0], 1, False, False),
    }
