"""ORACLE -- test infrastructure only.

Python face of the CPU restatement of carolc0708/graph-bit-ops' hot path
(oracle.cpp -> liboracle.so) plus pure-Python restatements of the two
Matrix Market readers.  Used by tests/ as the parity checker and by
bench.py's CPU-baseline legs; the product (libgbo) never imports it.

Tile words are exchanged as uint64 (one per b-bit word); `narrow()` casts
them to the reference's storage type for byte-exact comparisons.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
INF = 2147483647
WORD_DTYPE = {4: np.uint8, 8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}

_lib = None
_P = C.c_void_p
_I = C.c_int


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} missing: run make in {_HERE}")
        l = C.CDLL(LIB_PATH)
        sig = {
            "orc_pack_count": (C.c_longlong, [_P, _P, _I, _I, _P]),
            "orc_pack_fill": (None, [_P, _P, _I, _I, _I, _P, _P, _P]),
            "orc_pack_vector": (None, [_P, _I, _I, _P]),
            "orc_bmv_count": (None, [_P, _P, _P, _I, _I, _I, _P, _P]),
            "orc_bmv_masked": (None, [_P, _P, _P, _I, _I, _P, _P, _P]),
            "orc_bmv_minplus": (None, [_P, _P, _P, _I, _I, _I, _P, _P]),
            "orc_bmv_float": (None, [_P, _P, _P, _I, _I, _I, _P, _P, C.c_float, C.c_float, _P]),
            "orc_bmv_minselect": (None, [_P, _P, _P, _I, _I, _I, _P, _P]),
            "orc_bfs_b2sr": (_I, [_P, _P, _P, _I, _I, _I, _I, _P]),
            "orc_bfs_csr": (_I, [_P, _P, _I, _I, _P]),
            "orc_sssp_b2sr": (_I, [_P, _P, _P, _I, _I, _I, _I, _P]),
            "orc_pr_b2sr_f32": (_I, [_P, _P, _P, _I, _I, _I, _P, C.c_float, _I, C.c_float, _P]),
            "orc_pr_csr_f64": (_I, [_P, _P, _I, _P, C.c_double, _I, C.c_double, _P]),
            "orc_ppr_f64": (_I, [_P, _P, _I, _P, _P, C.c_double, C.c_double, _I, _P]),
            "orc_ppr_adjoint_f64": (_I, [_P, _P, _I, _P, _P, C.c_double, C.c_double, _I, _P]),
            "orc_cc": (None, [_P, _P, _I, _P]),
            "orc_verify_cc": (C.c_longlong, [_P, _P, _I, _P, C.POINTER(_I)]),
            "orc_tc_csr": (C.c_ulonglong, [_P, _P, _I]),
            "orc_tc_b2sr": (C.c_ulonglong, [_P, _P, _P, _I, _I]),
            "orc_spgemm_csr": (None, [_P, _P, _I, _P, _P, _I, _P, _P, _P]),
            "orc_bmm_sum_b2sr": (C.c_ulonglong, [_P, _P, _P, _I, _P, _P, _P, _I]),
            "orc_gen_rmat": (C.c_longlong, [_I, _I, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                            _P, _P]),
            "orc_bfs_shard_level": (C.c_ulonglong, [_P, _P, _I, _I, _P, _P, _P, _I, _P]),
            "orc_max_threads": (_I, []),
            "orc_set_threads": (None, [_I]),
        }
        for name, (res, args) in sig.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class B2SR:
    """CPU B2SR (words held as uint64)."""

    def __init__(self, rowptr, colind, words, nrows, ncols, b, layout=0):
        self.rowptr, self.colind, self.words = rowptr, colind, words
        self.nrows, self.ncols, self.b, self.layout = nrows, ncols, b, layout

    @property
    def nbr(self):
        return (self.nrows + self.b - 1) // self.b

    @property
    def nblk(self):
        return int(self.rowptr[-1])

    def narrow(self):
        return self.words.astype(WORD_DTYPE[self.b])


def pack(rowptr, colind, nrows, ncols, b, layout=0) -> B2SR:
    """csr2bsr_batch_{b} restated (algorithm/csr2bsr_batch_bsrbmv.cu)."""
    rowptr, colind = _i32(rowptr), _i32(colind)
    nbr = (nrows + b - 1) // b
    brp = np.zeros(nbr + 1, np.int32)
    nblk = lib().orc_pack_count(_p(rowptr), _p(colind), nrows, b, _p(brp))
    bci = np.zeros(max(1, nblk), np.int32)
    w = np.zeros(max(1, nblk * b), np.uint64)
    lib().orc_pack_fill(_p(rowptr), _p(colind), nrows, b, layout, _p(brp), _p(bci), _p(w))
    return B2SR(brp, bci[:nblk], w[: nblk * b], nrows, ncols, b, layout)


def pack_vector(x, b) -> np.ndarray:
    x = _i32(x)
    nw = (len(x) + b - 1) // b
    out = np.zeros(max(1, nw), np.uint64)
    lib().orc_pack_vector(_p(x), len(x), b, _p(out))
    return out[:nw]


def _g(g: B2SR):
    return _p(g.rowptr), _p(g.colind), _p(g.words), g.nbr, g.b


def _xpad(x, g: B2SR, dtype, fill=0):
    """Pad a per-vertex vector to whole tiles (ncols rounded up to b)."""
    nbc = (g.ncols + g.b - 1) // g.b
    out = np.full(max(nbc * g.b, len(x)), fill, dtype=dtype)
    out[: len(x)] = x
    return out


def bmv_count(g: B2SR, xwords) -> np.ndarray:
    nbc = (g.ncols + g.b - 1) // g.b
    xw = np.zeros(max(nbc, len(xwords)), np.uint64)
    xw[: len(xwords)] = xwords
    y = np.zeros(g.nrows, np.int32)
    lib().orc_bmv_count(*_g(g), g.nrows, _p(xw), _p(y))
    return y


def bmv_masked(g: B2SR, xwords, maskwords=None) -> np.ndarray:
    nbc = (g.ncols + g.b - 1) // g.b
    xw = np.zeros(max(nbc, len(xwords)), np.uint64)
    xw[: len(xwords)] = xwords
    out = np.zeros(max(1, g.nbr), np.uint64)
    mk = np.ascontiguousarray(maskwords, np.uint64) if maskwords is not None else None
    lib().orc_bmv_masked(*_g(g), _p(xw), _p(mk) if mk is not None else None, _p(out))
    return out[: g.nbr]


def bmv_minplus(g: B2SR, x) -> np.ndarray:
    xp = _xpad(np.asarray(x, np.uint32), g, np.uint32, INF)
    y = np.zeros(g.nrows, np.uint32)
    lib().orc_bmv_minplus(*_g(g), g.nrows, _p(xp), _p(y))
    return y


def bmv_float(g: B2SR, x, alpha=1.0, scale=None, add=0.0) -> np.ndarray:
    xp = _xpad(np.asarray(x, np.float32), g, np.float32)
    sp = _xpad(np.asarray(scale, np.float32), g, np.float32) if scale is not None else None
    y = np.zeros(g.nrows, np.float32)
    lib().orc_bmv_float(*_g(g), g.nrows, _p(xp), _p(sp) if sp is not None else None, alpha, add, _p(y))
    return y


def bmv_minselect(g: B2SR, x) -> np.ndarray:
    xp = _xpad(np.asarray(x, np.int32), g, np.int32, INF)
    y = np.zeros(g.nrows, np.int32)
    lib().orc_bmv_minselect(*_g(g), g.nrows, _p(xp), _p(y))
    return y


def bfs_b2sr(g: B2SR, src: int):
    lv = np.zeros(g.nrows, np.int32)
    d = lib().orc_bfs_b2sr(*_g(g), g.nrows, src, _p(lv))
    return lv, d


def bfs_csr(rowptr, colind, n, src):
    rowptr, colind = _i32(rowptr), _i32(colind)
    lv = np.zeros(n, np.int32)
    d = lib().orc_bfs_csr(_p(rowptr), _p(colind), n, src, _p(lv))
    return lv, d


def sssp_b2sr(g: B2SR, src: int):
    d = np.zeros(g.nrows, np.uint32)
    it = lib().orc_sssp_b2sr(*_g(g), g.nrows, src, _p(d))
    return d, it


def pagerank_b2sr_f32(g: B2SR, outdeg, alpha=0.85, max_iter=20, tol=-1.0):
    od = _xpad(_i32(outdeg), g, np.int32, 1)
    p = np.zeros(g.nrows, np.float32)
    it = lib().orc_pr_b2sr_f32(*_g(g), g.nrows, _p(od), alpha, max_iter, tol, _p(p))
    return p, it


def pagerank_f64(rowptr, colind, n, outdeg, alpha=0.85, max_iter=20, tol=-1.0):
    rowptr, colind, od = _i32(rowptr), _i32(colind), _i32(outdeg)
    p = np.zeros(n, np.float64)
    it = lib().orc_pr_csr_f64(_p(rowptr), _p(colind), n, _p(od), alpha, max_iter, tol, _p(p))
    return p, it


def ppr_f64(rowptr, colind, n, outdeg, v, alpha=0.85, tol=1e-12, max_iter=10000):
    rowptr, colind, od = _i32(rowptr), _i32(colind), _i32(outdeg)
    v = np.ascontiguousarray(v, np.float64)
    p = np.zeros(n, np.float64)
    it = lib().orc_ppr_f64(_p(rowptr), _p(colind), n, _p(od), _p(v), alpha, tol, max_iter, _p(p))
    return p, it


def ppr_adjoint_f64(rowptr, colind, n, outdeg, w, alpha=0.85, tol=1e-12, max_iter=10000):
    rowptr, colind, od = _i32(rowptr), _i32(colind), _i32(outdeg)
    w = np.ascontiguousarray(w, np.float64)
    g = np.zeros(n, np.float64)
    it = lib().orc_ppr_adjoint_f64(_p(rowptr), _p(colind), n, _p(od), _p(w), alpha, tol, max_iter,
                                   _p(g))
    return g, it


def cc(rowptr, colind, n):
    rowptr, colind = _i32(rowptr), _i32(colind)
    lab = np.zeros(n, np.int32)
    lib().orc_cc(_p(rowptr), _p(colind), n, _p(lab))
    return lab


def verify_cc(rowptr, colind, n, label):
    """SimpleVerifyCc (algorithm/cc.cu:21-60): (#mismatched edges, #components)."""
    rowptr, colind, label = _i32(rowptr), _i32(colind), _i32(label)
    nc = C.c_int(0)
    err = lib().orc_verify_cc(_p(rowptr), _p(colind), n, _p(label), C.byref(nc))
    return int(err), nc.value


def tc_csr(rowptr, colind, n) -> int:
    rowptr, colind = _i32(rowptr), _i32(colind)
    return int(lib().orc_tc_csr(_p(rowptr), _p(colind), n))


def tc_b2sr(lower: B2SR) -> int:
    return int(lib().orc_tc_b2sr(*_g(lower)))


def spgemm_csr(arp, aci, n, brp, bci, m):
    """C = A B over the integers (CSR in, CSR out: int64 rowptr, colind, counts)."""
    arp, aci, brp, bci = _i32(arp), _i32(aci), _i32(brp), _i32(bci)
    rowptr = np.zeros(n + 1, np.int64)
    lib().orc_spgemm_csr(_p(arp), _p(aci), n, _p(brp), _p(bci), m, _p(rowptr), None, None)
    rowptr = np.cumsum(rowptr).astype(np.int64)
    colind = np.zeros(max(1, int(rowptr[-1])), np.int32)
    val = np.zeros_like(colind)
    lib().orc_spgemm_csr(_p(arp), _p(aci), n, _p(brp), _p(bci), m, _p(rowptr), _p(colind), _p(val))
    nnz = int(rowptr[-1])
    return rowptr, colind[:nnz], val[:nnz]


def bmm_sum_b2sr(a: B2SR, b_col: B2SR) -> int:
    """Total of A B over tiles (A row words, B column words)."""
    assert a.b == b_col.b and b_col.layout == 1
    return int(lib().orc_bmm_sum_b2sr(_p(a.rowptr), _p(a.colind), _p(a.words), a.nbr,
                                      _p(b_col.rowptr), _p(b_col.colind), _p(b_col.words), a.b))


def bfs_shard_level(rowptr, colind, nrows, b, front, visited, level, lvl, nxt) -> int:
    """One pull level of a block-row BFS shard (uint64 words; visited, level
    and nxt are updated in place)."""
    rowptr, colind = _i32(rowptr), _i32(colind)
    return int(lib().orc_bfs_shard_level(_p(rowptr), _p(colind), nrows, b, _p(front), _p(visited),
                                         _p(level), lvl, _p(nxt)))


class Csr:
    """Host CSR (int32 rowptr / colind) made by the oracle's generators."""

    def __init__(self, rowptr, colind, nrows, ncols):
        self.rowptr, self.colind, self.nrows, self.ncols = rowptr, colind, nrows, ncols

    @property
    def nnz(self):
        return int(self.rowptr[-1])


def gen_rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=0) -> Csr:
    """The benchmark's R-MAT graph (symmetric, no self loops, deduplicated,
    rows sorted), built on the CPU without the product library."""
    n = 1 << scale
    rowptr = np.zeros(n + 1, np.int32)
    colind = np.empty(2 * n * edge_factor, np.int32)
    nnz = lib().orc_gen_rmat(scale, edge_factor, a, b, c, seed, _p(rowptr), _p(colind))
    return Csr(rowptr, colind[:nnz].copy(), n, n)


def set_threads(n: int):
    lib().orc_set_threads(n)


def max_threads() -> int:
    return lib().orc_max_threads()


# ------------------------------------------------- Matrix Market readers
def _parse_mtx(path):
    with open(path) as f:
        banner = f.readline().lower().split()
        line = f.readline()
        while line.startswith("%") or not line.strip():
            line = f.readline()
        nr, nc, nz = (int(t) for t in line.split()[:3])
        I, J = [], []
        for _ in range(nz):
            t = f.readline().split()
            I.append(int(t[0]) - 1)
            J.append(int(t[1]) - 1)
    sym = "symmetric" in banner and "skew-symmetric" not in banner
    herm = "hermitian" in banner
    return nr, nc, I, J, sym, herm


def _coo_to_csr(rows, cols, nrows):
    order = sorted(range(len(rows)), key=lambda k: (rows[k], cols[k]))
    rp = np.zeros(nrows + 1, np.int32)
    ci = np.zeros(len(rows), np.int32)
    for pos, k in enumerate(order):
        rp[rows[k] + 1] += 1
        ci[pos] = cols[k]
    return np.cumsum(rp).astype(np.int32), ci


def read_mtx_readmtx(path, directed=0, remove_self_loops=True):
    """readMtx + coo2csr (algorithm/readMtx.hpp:150-423, 246-304)."""
    nr, nc, I, J, sym, _ = _parse_mtx(path)
    undirected = sym or directed == 2
    if directed == 1:
        undirected = False
    rows, cols = list(I), list(J)
    if undirected:
        for i, j in zip(I, J):
            if i != j:
                rows.append(j)
                cols.append(i)
    pairs = sorted(set(zip(rows, cols)))
    if remove_self_loops:
        pairs = [(r, c) for r, c in pairs if r != c]
    return nr, nc, *_coo_to_csr([p[0] for p in pairs], [p[1] for p in pairs], nr)


def read_mtx_mmio(path):
    """mmio_data (algorithm/mmio_highlevel.h:139-309), rows sorted by column."""
    nr, nc, I, J, sym, herm = _parse_mtx(path)
    rows, cols = [], []
    for i, j in zip(I, J):
        rows.append(i)
        cols.append(j)
        if (sym or herm) and i != j:
            rows.append(j)
            cols.append(i)
    return nr, nc, *_coo_to_csr(rows, cols, nr)
