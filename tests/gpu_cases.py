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


def latehub(gbo, n=4096):
    """Rows whose only frontier neighbour is their last entry: a path
    0..50 then 4064; vertex 4000 is adjacent to 120 leaves in block columns
    4..123 (32-wide blocks) and to 4064 (block column 127), vertex 4002 to
    28 leaves and 4064; vertex 4001 is a hub of 100 leaves that the source
    never reaches.  With 32x32 tiles these rows hold 121, 29 and 100 row
    words, so the BFS pull scans long and short tails to their end."""
    src, dst = list(range(50)), list(range(1, 51))
    src.append(50)
    dst.append(4064)
    for i in range(120):
        src.append(4000)
        dst.append(128 + 32 * i)
    for i in range(28):
        src.append(4002)
        dst.append(130 + 32 * i)
    src += [4000, 4002]
    dst += [4064, 4064]
    for i in range(100):
        src.append(4001)
        dst.append(129 + 32 * i)
    return gbo.csr_from_edges(np.array(src, np.int32), np.array(dst, np.int32), n, True, True)


def cases(gbo):
    return {
        "er1000": gbo.gen_er(1000, 0.02002, 0),
        "rmat12": gbo.gen_rmat(12, 16, seed=0),
        "rmat14": gbo.gen_rmat(14, 8, seed=2),
        "mesh33": gbo.gen_king_mesh(33),
        "star20000": star(gbo, 20000),
        "ragged1001": ragged(gbo),
        "latehub": latehub(gbo),
        "single": gbo.csr_from_edges([0], [0], 1, False, False),
    }
