"""ctypes binding of libgbo (the C ABI in include/gbo.h) for Python callers.

This module is a thin host-side mirror of the C ABI: device buffers, the
graph handle, the B2SR primitives and the algorithms.  It contains no
computation of its own; every call goes to libgbo.so, and importing it on a
machine where libgbo.so is missing raises instead of falling back.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgbo.so")

GBO_OK = 0
GBO_ERR_INVALID = 1
GBO_ERR_CUDA = 2
GBO_ERR_NOMEM = 3
GBO_ERR_UNSORTED = 4
GBO_ERR_BOUNDS = 5
GBO_ERR_TIMEOUT = 6
GBO_ERR_IO = 7
GBO_ERR_UNSUPPORTED = 8
GBO_ERR_OVERFLOW = 9
GBO_ERR_NOTREADY = 10
GBO_ERR_FULL = 11
INJECT_HOST_ALLOC = 1
INJECT_REPLAY_CAP = 2
INJECT_SERVER_HOLD = 3
INJECT_BARRIER_SKIP = 4
BFS_LOOP_AUTO = 0
BFS_LOOP_GRAPH = 1
BFS_LOOP_COOP = 2

LAYOUT_ROW = 0
LAYOUT_COL = 1
FLAG_DEVICE_PTRS = 1
FLAG_TRANSPOSE = 2
FLAG_LAYOUT_COL = 4
FLAG_LOWER = 8
FLAG_SYMMETRIC = 16
FLAG_DEGREE_ORDER = 32
FLAG_TC_MMA = 64
OUT_I32 = 0
OUT_F32 = 1
MTX_READMTX = 0
MTX_MMIO = 1

WORD_DTYPE = {4: np.uint8, 8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}


class GboError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        super().__init__(f"{where}: {_status_name(status)}: {message}")
        self.status = status


class GraphInfo(C.Structure):
    _fields_ = [
        ("nrows", C.c_int), ("ncols", C.c_int), ("tile_bits", C.c_int), ("layout", C.c_int),
        ("nblockrows", C.c_int), ("nblockcols", C.c_int), ("nblocks", C.c_int64),
        ("nnz", C.c_int64), ("b2sr_bytes", C.c_int64), ("device_bytes", C.c_int64),
        ("nsplit_rows", C.c_int), ("nitems", C.c_int),
    ]


MAX_STEP_TIMES = 256


class RunStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("graph_replays", C.c_int),
                ("kernel_launches", C.c_longlong), ("nsteps", C.c_int),
                ("step_ms", C.c_float * MAX_STEP_TIMES)]


class ServerStats(C.Structure):
    _fields_ = [("rounds", C.c_longlong), ("bfs_completed", C.c_longlong),
                ("ppr_completed", C.c_longlong), ("kernel_launches", C.c_longlong),
                ("pending", C.c_longlong), ("in_flight", C.c_longlong),
                ("bfs_round_ms", C.c_double), ("ppr_round_ms", C.c_double),
                ("retire_ms", C.c_double), ("copy_ms", C.c_double), ("copy_wait_ms", C.c_double),
                ("copy_d2h_ms", C.c_double), ("copy_widen_ms", C.c_double)]


# Sharded BFS: the loop's operations and the data plane (include/gbo.h).
SHARD_LEVEL_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_uint64))
SHARD_ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_uint64))
SHARD_EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p)
SHARD_ALLGATHER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p)


class ShardOps(C.Structure):
    _fields_ = [("user", C.c_void_p), ("level", SHARD_LEVEL_FN), ("allreduce_sum_u64", SHARD_ALLREDUCE_FN),
                ("exchange", SHARD_EXCHANGE_FN)]


class ShardComm(C.Structure):
    _fields_ = [("user", C.c_void_p), ("allreduce_sum_u64", SHARD_ALLREDUCE_FN), ("allgather", SHARD_ALLGATHER_FN)]


class CsrStruct(C.Structure):
    _fields_ = [("nrows", C.c_int), ("ncols", C.c_int), ("nnz", C.c_int64),
                ("rowptr", C.POINTER(C.c_int)), ("colind", C.POINTER(C.c_int))]


_P = C.c_void_p
_I = C.c_int
_SIGS = {
    "gbo_status_string": (C.c_char_p, [_I]),
    "gbo_last_error": (C.c_char_p, []),
    "gbo_version": (_I, []),
    "gbo_device_count": (_I, [C.POINTER(_I)]),
    "gbo_set_device": (_I, [_I]),
    "gbo_malloc": (_I, [C.POINTER(_P), C.c_size_t]),
    "gbo_free": (_I, [_P]),
    "gbo_host_alloc": (_I, [C.POINTER(_P), C.c_size_t]),
    "gbo_host_free": (_I, [_P]),
    "gbo_memset": (_I, [_P, _I, C.c_size_t, _P]),
    "gbo_memcpy_h2d": (_I, [_P, _P, C.c_size_t, _P]),
    "gbo_memcpy_d2h": (_I, [_P, _P, C.c_size_t, _P]),
    "gbo_memcpy_d2d": (_I, [_P, _P, C.c_size_t, _P]),
    "gbo_stream_create": (_I, [C.POINTER(_P)]),
    "gbo_stream_destroy": (_I, [_P]),
    "gbo_stream_sync": (_I, [_P]),
    "gbo_device_sync": (_I, []),
    "gbo_event_create": (_I, [C.POINTER(_P)]),
    "gbo_event_destroy": (_I, [_P]),
    "gbo_event_record": (_I, [_P, _P]),
    "gbo_event_elapsed_ms": (_I, [_P, _P, C.POINTER(C.c_float)]),
    "gbo_flush_l2": (_I, [_P]),
    "gbo_b2sr_nnzb": (_I, [_P, _P, _I, _I, _I, _I, _P, C.POINTER(_I), _P]),
    "gbo_b2sr_pack": (_I, [_P, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P]),
    "gbo_pack_vector_f32": (_I, [_P, _I, _I, _P, _P]),
    "gbo_pack_vector_i32": (_I, [_P, _I, _I, _P, _P]),
    "gbo_unpack_vector": (_I, [_P, _I, _I, _P, _P]),
    "gbo_invdeg_from_rowptr": (_I, [_P, _I, _P, _P]),
    "gbo_graph_from_csr": (_I, [_P, _P, _I, _I, _I, _I, _I, _P, C.POINTER(_P)]),
    "gbo_graph_wrap_b2sr": (_I, [_I, _I, _I, _I, _I, _P, _P, _P, _P, _P, C.POINTER(_P)]),
    "gbo_graph_free": (_I, [_P]),
    "gbo_graph_save": (_I, [_P, C.c_char_p]),
    "gbo_graph_load": (_I, [C.c_char_p, _I, _P, C.POINTER(_P)]),
    "gbo_graph_get_info": (_I, [_P, C.POINTER(GraphInfo)]),
    "gbo_graph_b2sr": (_I, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
    "gbo_graph_outdeg": (_I, [_P, C.POINTER(_P)]),
    "gbo_graph_set_bfs_direction": (_I, [_P, _I, _I]),
    "gbo_graph_set_bfs_loop": (_I, [_P, _I, _I]),
    "gbo_graph_permutation": (_I, [_P, C.POINTER(_P)]),
    "gbo_tune_tile_width": (_I, [_P, _P, _I, _I, _I, _I, _I, _I, _P, C.POINTER(_I), _P]),
    "gbo_bmv_count": (_I, [_P, _P, _P, _I, _I, _P]),
    "gbo_bmv_count_noalloc": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _I, _I, _P]),
    "gbo_bmv_masked": (_I, [_P, _P, _P, _P, _P]),
    "gbo_bmv_minplus": (_I, [_P, _P, _P, _P]),
    "gbo_bmv_float": (_I, [_P, _P, _P, C.c_float, _P, C.c_float, _P]),
    "gbo_bmv_float_degptr": (_I, [_P, _P, _P, C.c_float, _P, _P]),
    "gbo_bmv_minselect": (_I, [_P, _P, _P, _P]),
    "gbo_bmv_float_transposed": (_I, [_P, _P, _P, C.c_float, _P, C.c_float, _P]),
    "gbo_bfs": (_I, [_P, _I, _P, C.POINTER(_I), _P]),
    "gbo_sssp_unit": (_I, [_P, _I, _P, C.POINTER(_I), _P]),
    "gbo_pagerank": (_I, [_P, C.c_float, _I, C.c_float, _P, C.POINTER(_I), _P]),
    "gbo_cc": (_I, [_P, _P, C.POINTER(_I), _P]),
    "gbo_tc": (_I, [_P, C.POINTER(C.c_uint64), _P]),
    "gbo_tc_device": (_I, [_P, _P, _P]),
    "gbo_ppr_forward": (_I, [_P, _P, C.c_float, C.c_float, _I, _P, C.POINTER(_I), _P]),
    "gbo_ppr_backward": (_I, [_P, _P, C.c_float, C.c_float, _I, _P, C.POINTER(_I), _P]),
    "gbo_graph_last_run": (_I, [_P, C.POINTER(RunStats)]),
    "gbo_msbfs": (_I, [_P, _P, _I, _P, C.POINTER(_I), _P]),
    "gbo_bfs_shard_level": (_I, [_P, _P, _P, _P, _I, _P, C.POINTER(C.c_uint64), _P]),
    "gbo_bfs_shard_loop": (_I, [_P, _I, C.POINTER(_I)]),
    "gbo_bfs_sharded": (_I, [_P, _I, _I, _P, _I, _P, C.POINTER(_I), _P, _P]),
    "gbo_nccl_unique_id": (_I, [_P]),
    "gbo_nccl_comm_create": (_I, [_I, _I, _P, C.POINTER(_P)]),
    "gbo_nccl_comm_destroy": (_I, [_P]),
    "gbo_bmm_sum": (_I, [_P, _P, C.POINTER(C.c_uint64), _P]),
    "gbo_spgemm_nnz": (_I, [_P, _P, _P, C.POINTER(C.c_int64), _P]),
    "gbo_spgemm_fill": (_I, [_P, _P, _P, _P, _P, _P]),
    "gbo_bfs_multi": (_I, [_P, _P, _I, _P, C.POINTER(_I), _P]),
    "gbo_server_create": (_I, [_P, _I, _I, C.c_float, C.c_float, _I, C.POINTER(_P)]),
    "gbo_server_set_queue_limit": (_I, [_P, C.c_longlong]),
    "gbo_server_set_admission": (_I, [_P, C.c_float]),
    "gbo_server_submit_bfs": (_I, [_P, _I, C.POINTER(C.c_int64)]),
    "gbo_server_submit_ppr": (_I, [_P, _P, _P, _I, C.POINTER(C.c_int64)]),
    "gbo_server_poll": (_I, [_P, C.c_int64, _P, C.POINTER(C.c_double), C.POINTER(_I)]),
    "gbo_server_wait": (_I, [_P, C.c_int64, _P, C.POINTER(C.c_double), C.POINTER(_I), C.c_double]),
    "gbo_server_wait_u8": (_I, [_P, C.c_int64, _P, C.POINTER(C.c_double), C.POINTER(_I), C.c_double]),
    "gbo_server_wait_device": (_I, [_P, C.c_int64, _P, C.POINTER(C.c_double), C.POINTER(_I),
                                    C.c_double, _P]),
    "gbo_server_get_stats": (_I, [_P, C.POINTER(ServerStats)]),
    "gbo_server_destroy": (_I, [_P]),
    "gbo_read_mtx": (_I, [C.c_char_p, _I, _I, C.POINTER(C.POINTER(CsrStruct))]),
    "gbo_csr_free": (_I, [C.POINTER(CsrStruct)]),
    "gbo_read_mtx_device": (_I, [C.c_char_p, _I, _I, C.POINTER(_P), C.POINTER(_P), C.POINTER(_I),
                                 C.POINTER(_I), C.POINTER(C.c_int64), _P]),
    "gbo_graph_from_mtx": (_I, [C.c_char_p, _I, _I, _I, _I, _P, C.POINTER(_P)]),
    "gbo_csr_transpose": (_I, [C.POINTER(CsrStruct), C.POINTER(C.POINTER(CsrStruct))]),
    "gbo_csr_tril": (_I, [C.POINTER(CsrStruct), C.POINTER(C.POINTER(CsrStruct))]),
    "gbo_csr_from_edges": (_I, [_P, _P, C.c_int64, _I, _I, _I, C.POINTER(C.POINTER(CsrStruct))]),
    "gbo_gen_rmat": (_I, [_I, _I, C.c_double, C.c_double, C.c_double, C.c_uint64,
                          C.POINTER(C.POINTER(CsrStruct))]),
    "gbo_gen_er": (_I, [_I, C.c_double, C.c_uint64, C.POINTER(C.POINTER(CsrStruct))]),
    "gbo_gen_er_avgdeg": (_I, [_I, C.c_double, C.c_uint64, C.POINTER(C.POINTER(CsrStruct))]),
    "gbo_gen_king_mesh": (_I, [_I, C.POINTER(C.POINTER(CsrStruct))]),
    "gbo_gen_er_batch": (_I, [_I, _I, _I, C.c_double, C.c_uint64, C.POINTER(C.POINTER(CsrStruct)), _P]),
    "gbo_debug_inject": (_I, [_I, C.c_longlong]),
}

_lib = None


def lib() -> C.CDLL:
    """Load libgbo.so (built by __graft_entry__.build() / make); raise if absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libgbo.so not found at {LIB_PATH}; run make in {_HERE}")
        l = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def exported_symbols():
    return list(_SIGS)


def _status_name(st: int) -> str:
    try:
        return lib().gbo_status_string(st).decode()
    except Exception:  # pragma: no cover - only while the library is unavailable
        return str(st)


def check(st: int, where: str = "gbo"):
    if st != GBO_OK:
        raise GboError(st, where, lib().gbo_last_error().decode())


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


# ------------------------------------------------------------ device memory
class DeviceBuffer:
    """Owned device allocation (gbo_malloc / gbo_free)."""

    def __init__(self, nbytes: int):
        self.nbytes = int(nbytes)
        p = C.c_void_p()
        check(lib().gbo_malloc(C.byref(p), max(1, self.nbytes)), "gbo_malloc")
        self.ptr = p.value

    @classmethod
    def from_numpy(cls, a: np.ndarray, stream=None) -> "DeviceBuffer":
        a = np.ascontiguousarray(a)
        buf = cls(a.nbytes)
        if a.nbytes:
            check(lib().gbo_memcpy_h2d(buf.ptr, _ptr(a), a.nbytes, stream), "h2d")
            check(lib().gbo_stream_sync(stream), "sync")
        return buf

    @classmethod
    def zeros(cls, nbytes: int, stream=None) -> "DeviceBuffer":
        buf = cls(nbytes)
        check(lib().gbo_memset(buf.ptr, 0, max(1, nbytes), stream), "memset")
        return buf

    def fill_bytes(self, value: int, stream=None):
        check(lib().gbo_memset(self.ptr, value, max(1, self.nbytes), stream), "memset")

    def upload(self, a: np.ndarray, stream=None):
        a = np.ascontiguousarray(a)
        assert a.nbytes <= self.nbytes
        if a.nbytes:
            check(lib().gbo_memcpy_h2d(self.ptr, _ptr(a), a.nbytes, stream), "h2d")

    def to_numpy(self, dtype, count: int | None = None, stream=None) -> np.ndarray:
        dtype = np.dtype(dtype)
        if count is None:
            count = self.nbytes // dtype.itemsize
        out = np.empty(count, dtype=dtype)
        if out.nbytes:
            check(lib().gbo_memcpy_d2h(_ptr(out), self.ptr, out.nbytes, stream), "d2h")
        check(lib().gbo_stream_sync(stream), "sync")
        return out

    def free(self):
        if self.ptr:
            lib().gbo_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def device_to_numpy(ptr: int, dtype, count: int, stream=None) -> np.ndarray:
    out = np.empty(count, dtype=np.dtype(dtype))
    if out.nbytes:
        check(lib().gbo_memcpy_d2h(_ptr(out), ptr, out.nbytes, stream), "d2h")
    check(lib().gbo_stream_sync(stream), "sync")
    return out


def debug_inject(what: int, n: int) -> None:
    """Fault injection (INJECT_*): host-side failures, or (INJECT_BARRIER_SKIP)
    a bounded device wait that runs out; n = 0 disarms."""
    check(lib().gbo_debug_inject(int(what), int(n)), "debug_inject")


def device_count() -> int:
    n = C.c_int(0)
    st = lib().gbo_device_count(C.byref(n))
    return n.value if st == GBO_OK else 0


def sync(stream=None):
    check(lib().gbo_stream_sync(stream), "sync")


class Stream:
    def __init__(self):
        p = C.c_void_p()
        check(lib().gbo_stream_create(C.byref(p)), "stream_create")
        self.ptr = p.value

    def sync(self):
        check(lib().gbo_stream_sync(self.ptr), "stream_sync")

    def __del__(self):
        try:
            if self.ptr:
                lib().gbo_stream_destroy(self.ptr)
        except Exception:
            pass


class Event:
    def __init__(self):
        p = C.c_void_p()
        check(lib().gbo_event_create(C.byref(p)), "event_create")
        self.ptr = p.value

    def record(self, stream=None):
        check(lib().gbo_event_record(self.ptr, stream), "event_record")

    def elapsed_ms(self, later: "Event") -> float:
        ms = C.c_float(0)
        check(lib().gbo_event_elapsed_ms(self.ptr, later.ptr, C.byref(ms)), "event_elapsed")
        return ms.value

    def __del__(self):
        try:
            if self.ptr:
                lib().gbo_event_destroy(self.ptr)
        except Exception:
            pass


# --------------------------------------------------------------- host CSR
class Csr:
    """Host CSR produced by libgbo (reader / generators); arrays are copied out."""

    def __init__(self, rowptr: np.ndarray, colind: np.ndarray, nrows: int, ncols: int):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.colind = np.ascontiguousarray(colind, dtype=np.int32)
        self.nrows = int(nrows)
        self.ncols = int(ncols)

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1]) if len(self.rowptr) else 0

    @classmethod
    def _take(cls, p) -> "Csr":
        s = p.contents
        n = s.nrows
        rp = np.ctypeslib.as_array(s.rowptr, shape=(n + 1,)).copy()
        ci = (np.ctypeslib.as_array(s.colind, shape=(int(s.nnz),)).copy()
              if s.nnz > 0 else np.zeros(0, np.int32))
        out = cls(rp, ci, n, s.ncols)
        lib().gbo_csr_free(p)
        return out

    def _struct(self):
        s = CsrStruct()
        s.nrows, s.ncols, s.nnz = self.nrows, self.ncols, self.nnz
        s.rowptr = self.rowptr.ctypes.data_as(C.POINTER(C.c_int))
        s.colind = self.colind.ctypes.data_as(C.POINTER(C.c_int))
        return s

    def transpose(self) -> "Csr":
        s = self._struct()
        out = C.POINTER(CsrStruct)()
        check(lib().gbo_csr_transpose(C.byref(s), C.byref(out)), "csr_transpose")
        return Csr._take(out)

    def tril(self) -> "Csr":
        s = self._struct()
        out = C.POINTER(CsrStruct)()
        check(lib().gbo_csr_tril(C.byref(s), C.byref(out)), "csr_tril")
        return Csr._take(out)

    def degrees(self) -> np.ndarray:
        return np.diff(self.rowptr)


def read_mtx_device(path: str, mode: int = MTX_READMTX, directed: int = 0) -> Csr:
    """gbo_read_mtx_device (parsed on the GPU); the CSR is copied back."""
    rp, ci = C.c_void_p(), C.c_void_p()
    nr, nc, nz = C.c_int(0), C.c_int(0), C.c_int64(0)
    check(lib().gbo_read_mtx_device(os.fsencode(path), mode, directed, C.byref(rp), C.byref(ci), C.byref(nr),
                                    C.byref(nc), C.byref(nz), None), "read_mtx_device")
    try:
        rowptr = device_to_numpy(rp.value, np.int32, nr.value + 1)
        colind = device_to_numpy(ci.value, np.int32, nz.value) if nz.value else np.zeros(0, np.int32)
    finally:
        lib().gbo_free(rp.value)
        lib().gbo_free(ci.value)
    return Csr(rowptr, colind, nr.value, nc.value)


def read_mtx(path: str, mode: int = MTX_READMTX, directed: int = 0) -> Csr:
    out = C.POINTER(CsrStruct)()
    check(lib().gbo_read_mtx(path.encode(), mode, directed, C.byref(out)), "read_mtx")
    return Csr._take(out)


def csr_from_edges(src, dst, nvertices: int, symmetrize=True, drop_self_loops=True) -> Csr:
    src = np.ascontiguousarray(src, dtype=np.int32)
    dst = np.ascontiguousarray(dst, dtype=np.int32)
    out = C.POINTER(CsrStruct)()
    check(lib().gbo_csr_from_edges(_ptr(src), _ptr(dst), len(src), nvertices, int(symmetrize),
                                   int(drop_self_loops), C.byref(out)), "csr_from_edges")
    return Csr._take(out)


def gen_rmat(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, seed: int = 0) -> Csr:
    out = C.POINTER(CsrStruct)()
    check(lib().gbo_gen_rmat(scale, edge_factor, a, b, c, seed, C.byref(out)), "gen_rmat")
    return Csr._take(out)


def gen_er(n: int, p: float, seed: int = 0) -> Csr:
    out = C.POINTER(CsrStruct)()
    check(lib().gbo_gen_er(n, p, seed, C.byref(out)), "gen_er")
    return Csr._take(out)


def gen_er_avgdeg(n: int, avg_degree: float, seed: int = 0) -> Csr:
    out = C.POINTER(CsrStruct)()
    check(lib().gbo_gen_er_avgdeg(n, avg_degree, seed, C.byref(out)), "gen_er_avgdeg")
    return Csr._take(out)


def gen_er_batch(count: int, nmin: int, nmax: int, avg_degree: float = 8.0, seed: int = 0):
    """Block-diagonal union of `count` ER graphs; returns (Csr, offsets)."""
    out = C.POINTER(CsrStruct)()
    off = np.zeros(count + 1, np.int32)
    check(lib().gbo_gen_er_batch(count, nmin, nmax, avg_degree, seed, C.byref(out), _ptr(off)),
          "gen_er_batch")
    return Csr._take(out), off


TUNE_BMV, TUNE_BFS, TUNE_TC = 0, 1, 2
TUNE_MODEL, TUNE_TIMED = 0, 1


def tune_tile_width(csr: "Csr", op: int = TUNE_BMV, mode: int = TUNE_MODEL, flags: int = 0, stream=None):
    """gbo_tune_tile_width: returns (best b, {b: bytes or ms})."""
    best = C.c_int(0)
    cost = np.zeros(5, np.float64)
    check(lib().gbo_tune_tile_width(_ptr(csr.rowptr), _ptr(csr.colind), csr.nrows, csr.ncols, csr.nnz,
                                    flags, op, mode, stream, C.byref(best), _ptr(cost)),
          "tune_tile_width")
    return best.value, dict(zip((4, 8, 16, 32, 64), cost.tolist()))


def gen_king_mesh(side: int) -> Csr:
    out = C.POINTER(CsrStruct)()
    check(lib().gbo_gen_king_mesh(side, C.byref(out)), "gen_king_mesh")
    return Csr._take(out)


# ------------------------------------------------------------ graph handle
class Graph:
    """Device-resident B2SR graph (gbo_graph_from_csr)."""

    def __init__(self, handle: int, keep=()):
        self.h = handle
        self._keep = keep  # buffers a wrapped graph points into

    @classmethod
    def from_csr(cls, csr: Csr, tile_bits: int = 32, flags: int = 0, stream=None) -> "Graph":
        p = C.c_void_p()
        check(lib().gbo_graph_from_csr(_ptr(csr.rowptr), _ptr(csr.colind), csr.nrows, csr.ncols,
                                       csr.nnz, tile_bits, flags, stream, C.byref(p)),
              "graph_from_csr")
        return cls(p.value)

    @classmethod
    def wrap_b2sr(cls, nrows, ncols, tile_bits, layout, nblocks, rowptr: DeviceBuffer,
                  colind: DeviceBuffer, val: DeviceBuffer, outdeg: DeviceBuffer | None = None,
                  stream=None) -> "Graph":
        p = C.c_void_p()
        check(lib().gbo_graph_wrap_b2sr(nrows, ncols, tile_bits, layout, nblocks, rowptr.ptr,
                                        colind.ptr, val.ptr, outdeg.ptr if outdeg else None,
                                        stream, C.byref(p)), "graph_wrap_b2sr")
        return cls(p.value, keep=(rowptr, colind, val, outdeg))

    @classmethod
    def from_mtx(cls, path: str, mode: int = MTX_READMTX, directed: int = 0, tile_bits: int = 32,
                 flags: int = 0, stream=None) -> "Graph":
        """Parse a Matrix Market file on the GPU and pack it (gbo_graph_from_mtx)."""
        p = C.c_void_p()
        check(lib().gbo_graph_from_mtx(os.fsencode(path), mode, directed, tile_bits, flags, stream, C.byref(p)),
              "graph_from_mtx")
        return cls(p.value)

    @classmethod
    def load(cls, path: str, flags: int = 0, stream=None) -> "Graph":
        """Rebuild a graph from a B2SR cache file written by save()."""
        p = C.c_void_p()
        check(lib().gbo_graph_load(os.fsencode(path), flags, stream, C.byref(p)), "graph_load")
        return cls(p.value)

    def save(self, path: str) -> None:
        """Write the B2SR arrays, out-degrees and permutation to a cache file."""
        check(lib().gbo_graph_save(self.h, os.fsencode(path)), "graph_save")

    def info(self) -> GraphInfo:
        inf = GraphInfo()
        check(lib().gbo_graph_get_info(self.h, C.byref(inf)), "graph_get_info")
        return inf

    def b2sr(self):
        """Copy the B2SR arrays back: (bsrRowPtr, bsrColInd, words)."""
        inf = self.info()
        r, c, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib().gbo_graph_b2sr(self.h, C.byref(r), C.byref(c), C.byref(v)), "graph_b2sr")
        nb = int(inf.nblocks)
        rp = device_to_numpy(r.value, np.int32, inf.nblockrows + 1)
        ci = device_to_numpy(c.value, np.int32, nb) if nb else np.zeros(0, np.int32)
        wd = WORD_DTYPE[inf.tile_bits]
        w = device_to_numpy(v.value, wd, nb * inf.tile_bits) if nb else np.zeros(0, wd)
        return rp, ci, w

    def outdeg(self) -> np.ndarray:
        p = C.c_void_p()
        check(lib().gbo_graph_outdeg(self.h, C.byref(p)), "graph_outdeg")
        return device_to_numpy(p.value, np.int32, self.info().ncols)

    def permutation(self):
        """new_of_old labels of a graph packed with FLAG_DEGREE_ORDER, else None."""
        p = C.c_void_p()
        check(lib().gbo_graph_permutation(self.h, C.byref(p)), "graph_permutation")
        return None if not p.value else device_to_numpy(p.value, np.int32, self.info().nrows)

    def set_bfs_direction(self, symmetric: bool, push_threshold: int = -1) -> None:
        """Allow top-down BFS steps on a symmetric graph below push_threshold
        frontier vertices (-1: nrows / 64; 0: pull only)."""
        check(lib().gbo_graph_set_bfs_direction(self.h, int(bool(symmetric)), push_threshold),
              "graph_set_bfs_direction")

    def set_bfs_loop(self, loop: int, coop_blocks: int = 0) -> None:
        """BFS level loop: BFS_LOOP_GRAPH (per-level kernels in a loop graph),
        BFS_LOOP_COOP (one cooperative launch, b = 32 ROW graphs) or
        BFS_LOOP_AUTO; coop_blocks > 0 sets the cooperative grid."""
        check(lib().gbo_graph_set_bfs_loop(self.h, int(loop), int(coop_blocks)), "graph_set_bfs_loop")

    def last_run(self) -> dict:
        st = RunStats()
        check(lib().gbo_graph_last_run(self.h, C.byref(st)), "graph_last_run")
        return {"iterations": st.iterations, "graph_replays": st.graph_replays,
                "kernel_launches": int(st.kernel_launches),
                "step_ms": [float(st.step_ms[i]) for i in range(st.nsteps)]}

    def free(self):
        if self.h:
            lib().gbo_graph_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    # ---- primitives on device buffers
    def bmv_count(self, x_bits: DeviceBuffer, y: DeviceBuffer, out_type=OUT_I32, accumulate=False,
                  stream=None):
        check(lib().gbo_bmv_count(self.h, x_bits.ptr, y.ptr, out_type, int(accumulate), stream),
              "bmv_count")

    def bmv_masked(self, x_bits: DeviceBuffer, mask_bits: DeviceBuffer | None, out_bits: DeviceBuffer,
                   stream=None):
        check(lib().gbo_bmv_masked(self.h, x_bits.ptr, mask_bits.ptr if mask_bits else None,
                                   out_bits.ptr, stream), "bmv_masked")

    def bmv_minplus(self, x: DeviceBuffer, y: DeviceBuffer, stream=None):
        check(lib().gbo_bmv_minplus(self.h, x.ptr, y.ptr, stream), "bmv_minplus")

    def bmv_float(self, x: DeviceBuffer, y: DeviceBuffer, alpha=1.0, scale: DeviceBuffer | None = None,
                  add=0.0, stream=None):
        check(lib().gbo_bmv_float(self.h, x.ptr, y.ptr, alpha, scale.ptr if scale else None, add,
                                  stream), "bmv_float")

    def bmv_minselect(self, x: DeviceBuffer, y: DeviceBuffer, stream=None):
        check(lib().gbo_bmv_minselect(self.h, x.ptr, y.ptr, stream), "bmv_minselect")

    def bmv_float_transposed(self, x: DeviceBuffer, y: DeviceBuffer, alpha=1.0,
                             scale: DeviceBuffer | None = None, add=0.0, stream=None):
        check(lib().gbo_bmv_float_transposed(self.h, x.ptr, y.ptr, alpha,
                                             scale.ptr if scale else None, add, stream),
              "bmv_float_transposed")

    # ---- algorithms (numpy in / numpy out helpers)
    def bfs(self, src: int, out: DeviceBuffer | None = None, stream=None, wait=True):
        """BFS levels from `src`: (levels, depth), or the depth when `out` is
        given.  wait=False (with `out`) queues the traversal and returns None
        at once (gbo_bfs with h_depth NULL)."""
        n = self.info().nrows
        buf = out or DeviceBuffer(4 * n)
        depth = C.c_int(0)
        if not wait and out is not None:
            check(lib().gbo_bfs(self.h, src, buf.ptr, None, stream), "bfs")
            return None
        check(lib().gbo_bfs(self.h, src, buf.ptr, C.byref(depth), stream), "bfs")
        if out is not None:
            return depth.value
        return buf.to_numpy(np.int32, n, stream), depth.value

    def msbfs(self, srcs, out: DeviceBuffer | None = None, stream=None):
        """Multi-source BFS; returns levels as an (n, k) int32 array (or the depth
        when `out` is given)."""
        srcs = np.ascontiguousarray(srcs, np.int32)
        n, k = self.info().nrows, len(srcs)
        buf = out or DeviceBuffer(4 * n * k)
        depth = C.c_int(0)
        check(lib().gbo_msbfs(self.h, _ptr(srcs), k, buf.ptr, C.byref(depth), stream), "msbfs")
        if out is not None:
            return depth.value
        return buf.to_numpy(np.int32, n * k, stream).reshape(n, k), depth.value

    def bfs_multi(self, seeds, out: DeviceBuffer | None = None, stream=None):
        seeds = np.ascontiguousarray(seeds, np.int32)
        n = self.info().nrows
        buf = out or DeviceBuffer(4 * n)
        depth = C.c_int(0)
        check(lib().gbo_bfs_multi(self.h, _ptr(seeds), len(seeds), buf.ptr, C.byref(depth), stream),
              "bfs_multi")
        if out is not None:
            return depth.value
        return buf.to_numpy(np.int32, n, stream), depth.value

    def sssp(self, src: int, stream=None):
        n = self.info().nrows
        buf = DeviceBuffer(4 * n)
        it = C.c_int(0)
        check(lib().gbo_sssp_unit(self.h, src, buf.ptr, C.byref(it), stream), "sssp_unit")
        return buf.to_numpy(np.uint32, n, stream), it.value

    def pagerank(self, alpha=0.85, max_iter=20, tol=-1.0, stream=None):
        n = self.info().nrows
        buf = DeviceBuffer(4 * n)
        it = C.c_int(0)
        check(lib().gbo_pagerank(self.h, alpha, max_iter, tol, buf.ptr, C.byref(it), stream),
              "pagerank")
        return buf.to_numpy(np.float32, n, stream), it.value

    def cc(self, stream=None):
        n = self.info().nrows
        buf = DeviceBuffer(4 * n)
        it = C.c_int(0)
        check(lib().gbo_cc(self.h, buf.ptr, C.byref(it), stream), "cc")
        return buf.to_numpy(np.int32, n, stream), it.value

    def bmm_sum(self, other: "Graph", stream=None) -> int:
        """Sum of all entries of self @ other over the integers."""
        out = C.c_uint64(0)
        check(lib().gbo_bmm_sum(self.h, other.h, C.byref(out), stream), "bmm_sum")
        return int(out.value)

    def spgemm(self, other: "Graph", stream=None):
        """self @ other (self: 32x32 ROW tiles, other: 32x32 COL tiles) as CSR:
        (int64 rowptr, int32 colind, int32 counts)."""
        n = self.info().nrows
        drp = DeviceBuffer(8 * (n + 1))
        nnz = C.c_int64(0)
        check(lib().gbo_spgemm_nnz(self.h, other.h, drp.ptr, C.byref(nnz), stream), "spgemm_nnz")
        m = int(nnz.value)
        dci, dv = DeviceBuffer(4 * max(m, 1)), DeviceBuffer(4 * max(m, 1))
        check(lib().gbo_spgemm_fill(self.h, other.h, drp.ptr, dci.ptr, dv.ptr, stream), "spgemm_fill")
        rp = drp.to_numpy(np.int64, n + 1, stream)
        if m == 0:
            return rp, np.zeros(0, np.int32), np.zeros(0, np.int32)
        return rp, dci.to_numpy(np.int32, m, stream), dv.to_numpy(np.int32, m, stream)

    def tc(self, stream=None) -> int:
        c = C.c_uint64(0)
        check(lib().gbo_tc(self.h, C.byref(c), stream), "tc")
        return int(c.value)

    def ppr_forward(self, v: np.ndarray, alpha=0.85, tol=1e-7, max_iter=1000, stream=None):
        n = self.info().nrows
        dv = DeviceBuffer.from_numpy(np.asarray(v, np.float32), stream)
        buf = DeviceBuffer(4 * n)
        it = C.c_int(0)
        check(lib().gbo_ppr_forward(self.h, dv.ptr, alpha, tol, max_iter, buf.ptr, C.byref(it),
                                    stream), "ppr_forward")
        return buf.to_numpy(np.float32, n, stream), it.value

    def ppr_backward(self, w: np.ndarray, alpha=0.85, tol=1e-7, max_iter=1000, stream=None):
        n = self.info().nrows
        dw = DeviceBuffer.from_numpy(np.asarray(w, np.float32), stream)
        buf = DeviceBuffer(4 * n)
        it = C.c_int(0)
        check(lib().gbo_ppr_backward(self.h, dw.ptr, alpha, tol, max_iter, buf.ptr, C.byref(it),
                                     stream), "ppr_backward")
        return buf.to_numpy(np.float32, n, stream), it.value


# ------------------------------------------------------------- raw B2SR
def b2sr_pack_raw(rowptr: DeviceBuffer, colind: DeviceBuffer, nrows, ncols, nnz, tile_bits,
                  layout=LAYOUT_ROW, stream=None):
    """gbo_b2sr_nnzb + gbo_b2sr_pack on caller-owned buffers; returns device buffers."""
    nbr = (nrows + tile_bits - 1) // tile_bits
    brp = DeviceBuffer(4 * (nbr + 1))
    nb = C.c_int(0)
    check(lib().gbo_b2sr_nnzb(rowptr.ptr, colind.ptr, nrows, ncols, nnz, tile_bits, brp.ptr,
                              C.byref(nb), stream), "b2sr_nnzb")
    wb = np.dtype(WORD_DTYPE[tile_bits]).itemsize
    bci = DeviceBuffer(4 * max(1, nb.value))
    val = DeviceBuffer(wb * tile_bits * max(1, nb.value))
    check(lib().gbo_b2sr_pack(rowptr.ptr, colind.ptr, nrows, ncols, nnz, tile_bits, layout, brp.ptr,
                              bci.ptr, val.ptr, stream), "b2sr_pack")
    return brp, bci, val, nb.value


def pack_vector(x: DeviceBuffer, n: int, tile_bits: int, dtype="f32", stream=None) -> DeviceBuffer:
    nw = (n + tile_bits - 1) // tile_bits
    wb = np.dtype(WORD_DTYPE[tile_bits]).itemsize
    out = DeviceBuffer(max(1, nw * wb))
    f = lib().gbo_pack_vector_f32 if dtype == "f32" else lib().gbo_pack_vector_i32
    check(f(x.ptr, n, tile_bits, out.ptr, stream), "pack_vector")
    return out


def bits_from_numpy(x01: np.ndarray, tile_bits: int) -> np.ndarray:
    """Host helper: 0/1 vector -> B2SR bit words (same layout as ToBit*Row)."""
    x01 = np.asarray(x01).astype(bool)
    n = len(x01)
    nw = (n + tile_bits - 1) // tile_bits
    pad = np.zeros(nw * tile_bits, dtype=bool)
    pad[:n] = x01
    bits = pad.reshape(nw, tile_bits).astype(np.uint64)
    weights = (np.uint64(1) << np.arange(tile_bits - 1, -1, -1, dtype=np.uint64))
    words = (bits * weights).sum(axis=1, dtype=np.uint64)
    return words.astype(WORD_DTYPE[tile_bits])


# ------------------------------------------------------------------ server
class Server:
    """Continuous-batching BFS / PPR query server over a resident graph."""

    def __init__(self, graph: Graph, bfs_slots=256, ppr_slots=32, alpha=0.85, tol=1e-7,
                 ppr_max_iter=1000):
        p = C.c_void_p()
        check(lib().gbo_server_create(graph.h, bfs_slots, ppr_slots, alpha, tol, ppr_max_iter,
                                      C.byref(p)), "server_create")
        self.h = p.value
        self.graph = graph
        self.n = graph.info().nrows

    def set_queue_limit(self, max_pending: int) -> None:
        """Submissions past max_pending queries not yet admitted return
        GBO_ERR_FULL (0: unbounded)."""
        check(lib().gbo_server_set_queue_limit(self.h, int(max_pending)), "server_set_queue_limit")

    def set_admission(self, min_free_fraction: float) -> None:
        """Pending BFS queries enter when at least this fraction of the slots
        is free or the engine is idle (0: every round, 1: batch after batch)."""
        check(lib().gbo_server_set_admission(self.h, C.c_float(min_free_fraction)), "server_set_admission")

    def submit_bfs(self, src: int) -> int:
        t = C.c_int64(0)
        check(lib().gbo_server_submit_bfs(self.h, int(src), C.byref(t)), "server_submit_bfs")
        return t.value

    def submit_ppr(self, verts, weights) -> int:
        v = np.ascontiguousarray(verts, np.int32)
        w = np.ascontiguousarray(weights, np.float32)
        t = C.c_int64(0)
        check(lib().gbo_server_submit_ppr(self.h, _ptr(v), _ptr(w), len(v), C.byref(t)),
              "server_submit_ppr")
        return t.value

    def wait(self, ticket: int, kind: str = "bfs", timeout=120.0, out: np.ndarray | None = None):
        """Block until the query's result is in host memory; `out` (n int32
        for BFS, n float32 for PPR) is reused when given."""
        if out is None:
            out = np.empty(self.n, np.int32 if kind == "bfs" else np.float32)
        lat, it = C.c_double(0), C.c_int(0)
        check(lib().gbo_server_wait(self.h, ticket, _ptr(out), C.byref(lat), C.byref(it), timeout),
              "server_wait")
        return out, lat.value, it.value

    def wait_u8(self, ticket: int, timeout=120.0, out=None):
        """BFS levels as uint8 (255 = unreachable): (levels, latency_ms,
        iterations).  `out` may be a uint8 array or a host pointer (int) of
        n bytes, e.g. pinned memory from gbo_host_alloc."""
        lat, it = C.c_double(0), C.c_int(0)
        if out is None:
            out = np.empty(self.n, np.uint8)
        ptr = out if isinstance(out, int) else _ptr(out)
        check(lib().gbo_server_wait_u8(self.h, ticket, ptr, C.byref(lat), C.byref(it), timeout), "server_wait_u8")
        return out, lat.value, it.value

    def wait_device(self, ticket: int, out, timeout=120.0):
        """Block until the query's result is in `out` (a DeviceBuffer of n
        int32 levels or n float32 PPR values); (latency_ms, iterations)."""
        lat, it = C.c_double(0), C.c_int(0)
        check(lib().gbo_server_wait_device(self.h, ticket, out.ptr, C.byref(lat), C.byref(it),
                                           timeout, None), "server_wait_device")
        return lat.value, it.value

    def poll(self, ticket: int, kind: str = "bfs"):
        """(result, latency_ms, iterations) or None while the query runs."""
        out = np.empty(self.n, np.int32 if kind == "bfs" else np.float32)
        lat, it = C.c_double(0), C.c_int(0)
        st = lib().gbo_server_poll(self.h, ticket, _ptr(out), C.byref(lat), C.byref(it))
        if st == GBO_ERR_NOTREADY:
            return None
        check(st, "server_poll")
        return out, lat.value, it.value

    def stats(self) -> dict:
        s = ServerStats()
        check(lib().gbo_server_get_stats(self.h, C.byref(s)), "server_get_stats")
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}

    def close(self):
        if self.h:
            lib().gbo_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
