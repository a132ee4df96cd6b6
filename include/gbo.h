/*
 * gbo.h -- C ABI of graph-bit-ops on B200 (sm_100a).
 *
 * The reference (carolc0708/graph-bit-ops) has no library: its drivers include
 * the kernel files textually and launch templated __global__ kernels on the
 * default stream.  This header is the drop-in boundary that replaces those
 * call sites.  Every entry point:
 *   - is extern "C", takes plain pointers and sizes, returns an int status;
 *   - is stream-ordered on the gbo_stream_t it is given (a cudaStream_t;
 *     NULL means the legacy default stream, as in the reference);
 *   - never calls exit(); on failure gbo_last_error() describes the cause.
 *
 * B2SR ("bit-packed BSR") layout, identical to the reference's:
 *   bsrRowPtr  int32[nblockrows+1]           ascending block-row offsets
 *   bsrColInd  int32[nblocks]                block columns, ascending per row
 *   bsrVal     nblocks * b words of b bits   word type per tile width b:
 *                b=4  uint8  (low nibble)    b=8  uint8
 *                b=16 uint16                 b=32 uint32     b=64 uint64
 *   ROW layout (GBO_LAYOUT_ROW): word r of a tile is tile row r and column c
 *     sits at bit (b-1-c)  -- cusparse DIRECTION_ROW + ToBit*Col
 *     (algorithm/bsrbmv.cu:31-235).
 *   COL layout (GBO_LAYOUT_COL): word c is tile column c and row r sits at
 *     bit (b-1-r)  -- the _col packers (bsrbmm/csr2bsr_batch.cu:1208).
 * Bit vectors use one word of the same type per block row; element
 * i = R*b + r is bit (b-1-r) of word R (ToBit*Row, algorithm/bsrbmv.cu:62-255).
 */
#ifndef GBO_H_
#define GBO_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
enum gbo_status {
  GBO_OK = 0,
  GBO_ERR_INVALID = 1,       /* bad argument (null pointer, size, tile width) */
  GBO_ERR_CUDA = 2,          /* a CUDA runtime call failed */
  GBO_ERR_NOMEM = 3,         /* device or host allocation failed */
  GBO_ERR_UNSORTED = 4,      /* CSR columns not ascending inside a row */
  GBO_ERR_BOUNDS = 5,        /* an index outside its range (device-checked) */
  GBO_ERR_TIMEOUT = 6,       /* a bounded device wait gave up */
  GBO_ERR_IO = 7,            /* file missing or malformed */
  GBO_ERR_UNSUPPORTED = 8,   /* combination not provided (e.g. layout) */
  GBO_ERR_OVERFLOW = 9,      /* a count does not fit the int32 B2SR indices */
  GBO_ERR_NOTREADY = 10,     /* server: result not yet available */
  GBO_ERR_FULL = 11          /* server: the admission queue is at its limit */
};

#if defined(__GNUC__)
#define GBO_API __attribute__((visibility("default")))
#else
#define GBO_API
#endif

typedef void* gbo_stream_t; /* cudaStream_t */

GBO_API const char* gbo_status_string(int status);
/* Message of the last failure on the calling host thread ("" if none). */
GBO_API const char* gbo_last_error(void);
GBO_API int gbo_version(void); /* major*10000 + minor*100 + patch */

enum { GBO_LAYOUT_ROW = 0, GBO_LAYOUT_COL = 1 };

/* ------------------------------------------- device plumbing for FFI users */
/* Thin wrappers so that callers without CUDA bindings (ctypes, cgo, JNI)
 * can own device buffers, streams and events.                              */
GBO_API int gbo_device_count(int* count);
GBO_API int gbo_set_device(int device);
GBO_API int gbo_malloc(void** d_ptr, size_t bytes);
GBO_API int gbo_free(void* d_ptr);
GBO_API int gbo_host_alloc(void** h_ptr, size_t bytes); /* pinned host memory */
GBO_API int gbo_host_free(void* h_ptr);
GBO_API int gbo_memset(void* d_ptr, int value, size_t bytes, gbo_stream_t stream);
GBO_API int gbo_memcpy_h2d(void* d_dst, const void* h_src, size_t bytes, gbo_stream_t stream);
GBO_API int gbo_memcpy_d2h(void* h_dst, const void* d_src, size_t bytes, gbo_stream_t stream);
GBO_API int gbo_memcpy_d2d(void* d_dst, const void* d_src, size_t bytes, gbo_stream_t stream);
GBO_API int gbo_stream_create(gbo_stream_t* stream);
GBO_API int gbo_stream_destroy(gbo_stream_t stream);
GBO_API int gbo_stream_sync(gbo_stream_t stream);
GBO_API int gbo_device_sync(void);
typedef void* gbo_event_t;
GBO_API int gbo_event_create(gbo_event_t* ev);
GBO_API int gbo_event_destroy(gbo_event_t ev);
GBO_API int gbo_event_record(gbo_event_t ev, gbo_stream_t stream);
GBO_API int gbo_event_elapsed_ms(gbo_event_t start, gbo_event_t stop, float* ms);
/* Write bytes >= the L2 size so the next timed launch starts cold. */
GBO_API int gbo_flush_l2(gbo_stream_t stream);

/* ------------------------------------------------ raw B2SR packing (A1, A2) */
/* Number of non-empty b x b tiles per block row of a CSR matrix.
 * Replaces cusparseXcsr2bsrNnz as used by the drivers (algorithm/bfs.cu:383).
 * d_bsrRowPtr gets nblockrows+1 offsets, *h_nblocks the total.
 * CSR column indices must be ascending inside each row (duplicates allowed);
 * otherwise GBO_ERR_UNSORTED.  All pointers are device pointers except
 * h_nblocks.  Synchronises the stream (the count sizes the next buffers). */
GBO_API int gbo_b2sr_nnzb(const int* d_csrRowPtr, const int* d_csrColInd, int nrows,
                  int ncols, int nnz, int tile_bits, int* d_bsrRowPtr,
                  int* h_nblocks, gbo_stream_t stream);

/* Fill bsrColInd / bsrVal for the offsets produced by gbo_b2sr_nnzb.
 * Replaces csr2bsr_batch_{4,8,16,32,64} (algorithm/csr2bsr_batch_bsrbmv.cu:
 * 9,180,406,621,786) and their _row/_col forms (bsrbmm/csr2bsr_batch.cu). */
GBO_API int gbo_b2sr_pack(const int* d_csrRowPtr, const int* d_csrColInd, int nrows,
                  int ncols, int nnz, int tile_bits, int layout,
                  const int* d_bsrRowPtr, int* d_bsrColInd, void* d_bsrVal,
                  gbo_stream_t stream);

/* Dense vector -> bit vector (element > 0 sets the bit); n_words words.
 * Replaces ToBit{4,8,16,32,64}Row (algorithm/bsrbmv.cu:62,110,154,195,239). */
GBO_API int gbo_pack_vector_f32(const float* d_x, int n, int tile_bits, void* d_bits,
                        gbo_stream_t stream);
GBO_API int gbo_pack_vector_i32(const int32_t* d_x, int n, int tile_bits, void* d_bits,
                        gbo_stream_t stream);
/* inv[i] = 1 / (rowptr[i+1] - rowptr[i]) (0 for empty rows), n entries: the
 * per-column scale the reference recomputes at every set bit
 * (algorithm/bsrbmv.cu:1277) precomputed once.  Device pointers. */
GBO_API int gbo_invdeg_from_rowptr(const int* d_rowptr, int n, float* d_inv,
                           gbo_stream_t stream);
/* Bit vector -> int32 0/1 per element (n elements). */
GBO_API int gbo_unpack_vector(const void* d_bits, int n, int tile_bits, int32_t* d_out,
                      gbo_stream_t stream);

/* ----------------------------------------------------------- graph handle */
typedef struct gbo_graph gbo_graph;

enum gbo_graph_flags {
  GBO_FLAG_DEVICE_PTRS = 1, /* rowptr/colind are device pointers (else host) */
  GBO_FLAG_TRANSPOSE = 2,   /* pack the transpose of the given CSR (CSC) */
  GBO_FLAG_LAYOUT_COL = 4,  /* COL tile layout instead of ROW */
  GBO_FLAG_LOWER = 8,       /* keep only row >= col entries (tril_csr) */
  GBO_FLAG_SYMMETRIC = 16,  /* caller asserts the packed matrix is symmetric:
                               BFS may then take top-down (push) steps while
                               the frontier is small (direction-optimising) */
  GBO_FLAG_DEGREE_ORDER = 32, /* relabel vertices by descending degree before
                               packing (P' = Q P Q^T; gbo_graph_permutation
                               gives the labels).  For permutation-invariant
                               results such as the triangle count: with
                               GBO_FLAG_LOWER every row then holds only
                               higher-degree neighbours, so hub rows stay
                               short.  No reference counterpart. */
  GBO_FLAG_TC_MMA = 64       /* b = 32: count the mask tiles with more than 16
                               bits on the 1-bit tensor-core MMA
                               (mma.sync m16n8k256 AND-popc, 8 hits per
                               step).  Opt-in: on sparse-tile graphs the
                               CUDA-core path is as fast or faster. */
};

/* Pack a CSR matrix M into a device-resident B2SR graph owned by the handle.
 * The algorithms below treat the packed matrix P as a pull operator:
 * y[i] = (+)_{j : P[i][j] = 1} x[j].  The reference packs the CSC of A
 * (algorithm/bfs.cu:398-423) so that BFS pulls along A's edges; pass
 * GBO_FLAG_TRANSPOSE to get the same.  out-degrees (column counts of P
 * including duplicate CSR entries, i.e. the reference's csrRowPtr deltas
 * used at algorithm/bsrbmv.cu:1277) are kept for PageRank. */
GBO_API int gbo_graph_from_csr(const int* rowptr, const int* colind, int nrows,
                       int ncols, int nnz, int tile_bits, int flags,
                       gbo_stream_t stream, gbo_graph** out);
/* Wrap caller-owned device B2SR buffers (not copied, not freed).  d_outdeg
 * may be NULL (then PageRank entry points return GBO_ERR_INVALID).  The
 * work schedule and, for 32x32 ROW tiles, the per-tile occupancy words and
 * packed non-empty row words are derived from the buffers here, so their
 * contents must not change while the graph is in use. */
GBO_API int gbo_graph_wrap_b2sr(int nrows, int ncols, int tile_bits, int layout,
                        int nblocks, const int* d_bsrRowPtr,
                        const int* d_bsrColInd, const void* d_bsrVal,
                        const int* d_outdeg, gbo_stream_t stream,
                        gbo_graph** out);
GBO_API int gbo_graph_free(gbo_graph* g);
/* Binary B2SR cache file.  gbo_graph_save writes g's B2SR arrays (the
 * reference layout, byte for byte), its out-degrees and its vertex
 * permutation (GBO_FLAG_DEGREE_ORDER) to `path`; gbo_graph_load rebuilds the
 * graph from such a file without reparsing or repacking (flags:
 * GBO_FLAG_SYMMETRIC, GBO_FLAG_TC_MMA as in gbo_graph_from_csr; a graph
 * saved as symmetric stays symmetric).  Malformed files return GBO_ERR_IO.
 * No reference counterpart: the reference reads the .mtx and repacks on
 * every run (algorithm/bfs.cu:333-424). */
GBO_API int gbo_graph_save(const gbo_graph* g, const char* path);
GBO_API int gbo_graph_load(const char* path, int flags, gbo_stream_t stream,
                   gbo_graph** out);

typedef struct gbo_graph_info {
  int nrows, ncols, tile_bits, layout;
  int nblockrows, nblockcols;
  int64_t nblocks;
  int64_t nnz;          /* CSR entries the graph was packed from (-1 if wrapped) */
  int64_t b2sr_bytes;   /* rowptr + colind + tile words */
  int64_t device_bytes; /* everything the handle owns on the device */
  int nsplit_rows;      /* block rows split across warps for load balance */
  int nitems;           /* warp work items of the balanced schedule */
} gbo_graph_info;
GBO_API int gbo_graph_get_info(const gbo_graph* g, gbo_graph_info* info);
GBO_API int gbo_graph_b2sr(const gbo_graph* g, const int** d_bsrRowPtr,
                   const int** d_bsrColInd, const void** d_bsrVal);
/* Device array of out-degrees (ncols ints) or NULL. */
GBO_API int gbo_graph_outdeg(const gbo_graph* g, const int** d_outdeg);
/* Device array new_of_old[v] (nrows ints) of a graph packed with
 * GBO_FLAG_DEGREE_ORDER, else NULL. */
GBO_API int gbo_graph_permutation(const gbo_graph* g, const int** d_new_of_old);
/* Direction-optimising BFS control (no counterpart in the reference, whose
 * BFS only pulls).  symmetric = 1 asserts P == P^T (what GBO_FLAG_SYMMETRIC
 * does for gbo_graph_from_csr; needed for wrapped graphs), 0 restores
 * pull-only BFS.  A level whose frontier holds fewer than push_threshold
 * vertices is expanded top-down; -1 selects the default nrows / 64.
 * gbo_msbfs on a symmetric graph pushes a level with fewer than
 * push_threshold new (vertex, source) pairs when push_threshold > 0 (any k
 * on b = 32 ROW graphs, k <= 64 on others), and otherwise (-1 and 0) pulls
 * every level, except that level 0 on a b = 32 ROW graph pushes from the
 * sources.
 * Rejected (GBO_ERR_UNSUPPORTED) for a non-square graph. */
GBO_API int gbo_graph_set_bfs_direction(gbo_graph* g, int symmetric, int push_threshold);

/* How gbo_bfs / gbo_bfs_multi / gbo_sssp run their level loop (no
 * counterpart in the reference, whose BFS loop copies a flag to the host
 * after every level).
 *   GBO_BFS_LOOP_GRAPH: the level's kernels (pull, push, finish) in a CUDA
 *     graph whose conditional WHILE node repeats them until a level adds no
 *     vertex; every graph.
 *   GBO_BFS_LOOP_COOP: the whole loop in one cooperative launch whose blocks
 *     meet at a grid barrier after each level; b = 32 ROW graphs only
 *     (GBO_ERR_UNSUPPORTED otherwise).  coop_blocks > 0 sets its grid (capped
 *     at the blocks that fit on the device at once), 0 sizes it by the graph.
 *     A barrier that waits longer than 5 s gives up: the call returns
 *     GBO_ERR_TIMEOUT (synchronous form) and the levels are incomplete.
 *   GBO_BFS_LOOP_AUTO (the default): GBO_BFS_LOOP_COOP where it applies,
 *     else GBO_BFS_LOOP_GRAPH.
 * Both loops give the same levels. */
enum { GBO_BFS_LOOP_AUTO = 0, GBO_BFS_LOOP_GRAPH = 1, GBO_BFS_LOOP_COOP = 2 };
GBO_API int gbo_graph_set_bfs_loop(gbo_graph* g, int loop, int coop_blocks);

/* Tile-width tuner (no counterpart in the reference, whose drivers take b
 * from the command line).  Ranks b = 4, 8, 16, 32, 64 for the CSR matrix
 * (same arguments and flags as gbo_graph_from_csr) and an operation:
 *   mode GBO_TUNE_MODEL: algorithmic bytes of one sweep over the packing
 *     (nblocks(b) * (b words + 4-byte column index) + block-row offsets;
 *     for GBO_TUNE_BFS at b = 32 in the ROW layout, the row-word slices that
 *     its BFS walks: 8 bytes per non-empty row word + 8 per row), from count
 *     passes only -- nothing is packed.  A BFS reads less than one sweep
 *     (pull steps stop at a row's first frontier neighbour), so
 *     GBO_TUNE_TIMED ranks BFS widths more faithfully;
 *   mode GBO_TUNE_TIMED: packs at every width and times the operation
 *     (one warm-up, mean of three runs, CUDA events on `stream`).
 * op GBO_TUNE_TC packs the lower triangle and never picks b = 4.
 * *best_bits gets the cheapest width; cost (nullable, 5 doubles, widths in
 * the order above) gets bytes or milliseconds (INFINITY where a width
 * overflows the int32 tile count). */
enum { GBO_TUNE_BMV = 0, GBO_TUNE_BFS = 1, GBO_TUNE_TC = 2 };
enum { GBO_TUNE_MODEL = 0, GBO_TUNE_TIMED = 1 };
GBO_API int gbo_tune_tile_width(const int* rowptr, const int* colind, int nrows, int ncols,
                                int nnz, int flags, int op, int mode, gbo_stream_t stream,
                                int* best_bits, double* cost);

/* ------------------------------------------------ BMV primitives (A3-A8) */
enum { GBO_OUT_I32 = 0, GBO_OUT_F32 = 1 };
/* y[i] (+)= popc over tiles of (P_row_i & x) = sum_j P[i][j]*x[j]  (exact).
 * y has nrows entries of type out_type; accumulate=1 adds to y like the
 * reference's "+=" (bsrbmv.cu:432), 0 overwrites.
 * Replaces bmv{4,8,16,32,64}_sparse and *_sparse_new (bsrbmv.cu:262-474,
 * 2434-3094).  Unlike the reference b=64 kernel (16-bit halves,
 * bsrbmv.cu:464-471) counts are exact 32-bit. */
GBO_API int gbo_bmv_count(const gbo_graph* g, const void* d_x_bits, void* d_y,
                  int out_type, int accumulate, gbo_stream_t stream);
/* The same y as gbo_bmv_count, computed straight from caller-owned ROW-layout
 * B2SR arrays (bsrRowPtr: ceil(nrows/b)+1 ints ending at nblocks; bsrColInd,
 * bsrVal as gbo_b2sr_pack writes them) without a graph handle, and without
 * allocating any device or host memory at any call.  No counterpart in the
 * reference.  For callers that may not allocate: a framework that owns all
 * device memory through its own pool, or a thread that must not let
 * cudaMalloc / cudaFree synchronise a device shared with other streams.
 * Row partials of long block rows go to one fixed 8 MiB device array inside
 * this library, shared by every call on a device:
 *   - at most 2^35 / b^2 tiles per call (33,554,432 at b = 32, 8,388,608 at
 *     b = 64); more returns GBO_ERR_UNSUPPORTED before any launch;
 *   - calls whose kernels may overlap (other streams, unordered threads)
 *     race on that array and can return wrong counts: order them;
 *   - the first call on each device looks up the array's device address
 *     (cudaGetSymbolAddress, which may load this library's device code):
 *     make that first call before any stream capture begins;
 *   - the row pointer is not validated on the device (that would need a
 *     read back): a malformed one (not non-decreasing from 0 to nblocks)
 *     leaves y undefined. */
GBO_API int gbo_bmv_count_noalloc(int nrows, int ncols, int tile_bits, int nblocks,
                                  const int* d_bsrRowPtr, const int* d_bsrColInd,
                                  const void* d_bsrVal, const void* d_x_bits, void* d_y,
                                  int out_type, int accumulate, gbo_stream_t stream);
/* out_bits[R] = bits (sum_j P[i][j] x[j] > 0) & ~mask[R]  (Boolean OR.AND with
 * a complement mask).  Replaces bmv32_sparse_bin_masked_v4 and
 * bmv4_sparse_bin_masked_v4 (bsrbmv.cu:637-783).  d_mask_bits may be NULL. */
GBO_API int gbo_bmv_masked(const gbo_graph* g, const void* d_x_bits,
                   const void* d_mask_bits, void* d_out_bits,
                   gbo_stream_t stream);
/* y[i] = min(x[i], min_{j: P[i][j]} x[j] (+) 1) over uint32 with
 * 2147483647 as infinity (saturating).  The min-plus product of (P + I),
 * bmv{4,32}_sparse_full_minplus (bsrbmv.cu:989-1138). */
GBO_API int gbo_bmv_minplus(const gbo_graph* g, const uint32_t* d_x, uint32_t* d_y,
                    gbo_stream_t stream);
/* y[i] = alpha * sum_{j: P[i][j]} x[j] * scale[j] + add   (fp32).
 * scale may be NULL (1).  bmv{4,32}_sparse_full (bsrbmv.cu:1156-1286) is
 * scale = 1/outdeg, add = 0. */
GBO_API int gbo_bmv_float(const gbo_graph* g, const float* d_x, float* d_y,
                  float alpha, const float* d_scale, float add,
                  gbo_stream_t stream);
/* The reference's own form of the fp32 BMV: y[i] = alpha * sum_{j: P[i][j]}
 * x[j] / (csrRowPtr[j+1] - csrRowPtr[j]), the degree read from a CSR row
 * pointer only at set bits (bmv32_sparse_full, algorithm/bsrbmv.cu:1239-1286,
 * which writes C = sum; the caller adds (1-alpha)/n, pr.cu:486). */
GBO_API int gbo_bmv_float_degptr(const gbo_graph* g, const float* d_x, float* d_y,
                         float alpha, const int* d_csrRowPtr,
                         gbo_stream_t stream);
/* y[i] = min_{j: P[i][j]} x[j], INT32_MAX when row i is empty.
 * bmv{4,8,16,32}_sparse_full_cc* (bsrbmv.cu:1367-2099). */
GBO_API int gbo_bmv_minselect(const gbo_graph* g, const int32_t* d_x, int32_t* d_y,
                      gbo_stream_t stream);
/* y[j] = alpha * sum_{i: P[i][j]} x[i] * scale[i] + add  (y = alpha P^T x):
 * the transposed bit-packed BMV used by the PageRank adjoint.  No reference
 * counterpart; fp32 with atomics, ncols outputs. */
GBO_API int gbo_bmv_float_transposed(const gbo_graph* g, const float* d_x, float* d_y,
                             float alpha, const float* d_scale, float add,
                             gbo_stream_t stream);

/* --------------------------------------------------- algorithms (A5-A11) */
/* Level-synchronous pull BFS on P from src: level[i] = hops, -1 unreachable.
 * Rewrites algorithm/bfs.cu:508-564 with all state on the device and
 * termination decided on the device (no per-level host copy).
 * h_depth (nullable) receives the number of levels (max level + 1); the
 * call then waits for the traversal.  With h_depth NULL it is asynchronous:
 * the whole level loop runs on the device (one CUDA graph with a device-side
 * loop) and the call returns once it is queued on `stream`.
 * Takes ROW- and COL-layout graphs (the other algorithms need ROW): with
 * column words a pull step reads, per tile, only the words of the
 * frontier's columns, which pays off where frontier segments are sparse in
 * dense tiles; on sparse tiles (R-MAT) the 32-byte DRAM sectors make both
 * layouts read about the same bytes and ROW is faster. */
GBO_API int gbo_bfs(const gbo_graph* g, int src, int32_t* d_level, int* h_depth,
            gbo_stream_t stream);
/* Unit-weight SSSP with the distances of the reference's min-plus loop
 * (algorithm/sssp.cu:420-470): dist[i] in uint32, 2147483647 = unreachable.
 * With unit weights every frontier vertex at iteration k has distance k, so
 * a row's relaxation min_j (d[j] + 1) is k + 1 at its first frontier
 * neighbour: the step runs as the BFS step (early exit; push on small
 * frontiers of symmetric graphs).  The general min-plus product is
 * gbo_bmv_minplus. */
GBO_API int gbo_sssp_unit(const gbo_graph* g, int src, uint32_t* d_dist, int* h_iters,
                  gbo_stream_t stream);
/* PageRank p = alpha * P D^-1 p + (1-alpha)/n from p0 = 1/n, as in
 * algorithm/pr.cu:449-513 (no dangling redistribution; D = out-degrees).
 * Runs until ||p - p_prev||_2 <= tol or max_iter iterations (tol < 0 runs
 * exactly max_iter).  *h_iters gets the iterations done. */
GBO_API int gbo_pagerank(const gbo_graph* g, float alpha, int max_iter, float tol,
                 float* d_p, int* h_iters, gbo_stream_t stream);
/* Connected components (P symmetric): label[i] = smallest vertex id in the
 * component of i -- the fixed point of the reference's FastSV loop
 * (algorithm/cc.cu:223-287). */
GBO_API int gbo_cc(const gbo_graph* g, int32_t* d_label, int* h_iters,
           gbo_stream_t stream);
/* Triangles of an undirected simple graph given its lower triangle L
 * (graph built with GBO_FLAG_LOWER, ROW layout): sum over (i,k) in L of
 * (L L^T)[i][k].  Replaces tril_csr + bmm*_sparse_masked_v5 with a uint64
 * result (bsrbmm/bsrbmm.cu:1214-1265, 1416; bsrbmm/tc.cu:767-951). */
GBO_API int gbo_tc(const gbo_graph* lower, uint64_t* h_count, gbo_stream_t stream);
/* Same, result left in device memory (*d_count is overwritten). */
GBO_API int gbo_tc_device(const gbo_graph* lower, unsigned long long* d_count,
                  gbo_stream_t stream);

/* Unmasked products (bsrbmm/bsrbmm.cu:244-555, bmm{4..64}_sparse): the sum
 * of all entries of A B over the integers (A.ncols == B.nrows, same tile
 * width, either layout), computed as sum_m colcount_A(m) * rowcount_B(m). */
GBO_API int gbo_bmm_sum(const gbo_graph* a, const gbo_graph* b, uint64_t* h_sum,
                gbo_stream_t stream);
/* Sparse-output product C = A B over the integers (bsrbmm/bsrbmm.cu:
 * 1273-1373, bmm32_sparse_symbolic/numeric): A with 32x32 ROW tiles, B with
 * 32x32 COL tiles (as the reference packs it).  C is CSR with int64 row
 * offsets, columns ascending in each row, and values C[i][j] = number of k
 * with A[i][k] = B[k][j] = 1 (zeros not stored).  Two passes: gbo_spgemm_nnz
 * writes d_rowptr[A.nrows + 1] and the entry count; the caller allocates
 * d_colind and d_val (int32[nnz]) for gbo_spgemm_fill. */
GBO_API int gbo_spgemm_nnz(const gbo_graph* a, const gbo_graph* b, int64_t* d_rowptr,
                   int64_t* h_nnz, gbo_stream_t stream);
GBO_API int gbo_spgemm_fill(const gbo_graph* a, const gbo_graph* b,
                    const int64_t* d_rowptr, int32_t* d_colind, int32_t* d_val,
                    gbo_stream_t stream);

/* Block-row sharding of BFS across GPUs (the reference runs on one GPU,
 * algorithm/bfs.cu:508-564 is its level loop).  A shard is a graph packed
 * from the CSR rows [row0, row0 + shard.nrows) of the whole matrix with all
 * of its columns (row0 a multiple of the tile width, ROW layout).  One call
 * runs one pull level over the shard:
 *   d_front   the whole graph's frontier words of `level` (ncols/b words, the
 *             bit-vector layout of gbo_pack_vector_*),
 *   d_visited the shard's visited words (updated), d_level the shard's int32
 *             levels (new vertices get level + 1), d_next the shard's
 *             next-frontier words (written), *h_count (may be NULL) the
 *             number of new vertices (the call then waits for the stream).
 * Between levels every rank places the shards' d_next words at their block
 * rows to form the next d_front (an all-gather of n/8 bytes); the loop ends
 * when no shard finds a new vertex.  gbo_bfs_sharded (below) runs that loop. */
GBO_API int gbo_bfs_shard_level(const gbo_graph* shard, const void* d_front, void* d_visited,
                        int32_t* d_level, int level, void* d_next, uint64_t* h_count,
                        gbo_stream_t stream);

/* The level loop of a block-row sharded BFS over caller-supplied operations
 * (one rank; every rank of the job calls it):
 *   level(user, L, &count)     one pull level of this rank's shard against the
 *                              frontier of level L; count = its new vertices
 *   allreduce_sum_u64(user, &v) v summed over all ranks, in place (host)
 *   exchange(user)             every rank's next-frontier words into every
 *                              rank's frontier of the next level
 * The loop stops when the summed count is 0 (*h_depth = levels) or after
 * max_levels levels (GBO_ERR_TIMEOUT).  A rank whose level step fails adds
 * an error mark to the sum instead of its count, so all ranks leave at the
 * same level with the same error.  gbo_bfs_sharded runs it on the GPU; the
 * operations can also be a CPU step over any transport (the tests run it
 * over gloo).  The reference has no multi-GPU path (its loop is
 * algorithm/bfs.cu:508-564). */
typedef struct gbo_shard_ops {
  void* user;
  int (*level)(void* user, int level, uint64_t* new_vertices);
  int (*allreduce_sum_u64)(void* user, uint64_t* value);
  int (*exchange)(void* user);
} gbo_shard_ops;
GBO_API int gbo_bfs_shard_loop(const gbo_shard_ops* ops, int max_levels, int* h_depth);

/* The data plane of a sharded BFS: a sum of one host uint64 over all ranks,
 * and an all-gather of `bytes` device bytes per rank (rank r's bytes at
 * d_recv + r * bytes) on `stream`.  gbo_nccl_comm_create makes one over
 * NCCL (NVLink / NVSwitch between GPUs); callers may supply their own. */
typedef struct gbo_shard_comm {
  void* user;
  int (*allreduce_sum_u64)(void* user, uint64_t* value);
  int (*allgather)(void* user, const void* d_send, void* d_recv, size_t bytes, gbo_stream_t stream);
} gbo_shard_comm;
/* BFS from src over all ranks, this rank holding rows [h_bounds[rank],
 * h_bounds[rank+1]) of an n = h_bounds[world] vertex graph (every column;
 * bounds on tile boundaries, e.g. balanced by stored entries) as `shard`.
 * d_level gets the int32 levels of the shard's rows (-1 unreachable), every
 * rank *h_depth.  Allocates its frontier and exchange buffers on `stream`
 * (stream-ordered) for the call; returns after the stream has finished. */
GBO_API int gbo_bfs_sharded(const gbo_graph* shard, int rank, int world, const int* h_bounds, int src,
                            int32_t* d_level, int* h_depth, const gbo_shard_comm* comm,
                            gbo_stream_t stream);
/* NCCL data plane: gbo_nccl_unique_id fills 128 bytes on one rank, which
 * the caller hands to every rank (any host channel); each rank then makes
 * its communicator (its CUDA device current).  NCCL is loaded at run time
 * (libnccl.so.2): GBO_ERR_UNSUPPORTED without it. */
GBO_API int gbo_nccl_unique_id(void* h_id128);
GBO_API int gbo_nccl_comm_create(int world, int rank, const void* h_id128, gbo_shard_comm** out);
GBO_API int gbo_nccl_comm_destroy(gbo_shard_comm* comm);

/* Multi-source BFS (batching): k sources (1 <= k <= 1024) traversed at once.
 * The frontier is an n x k bit matrix, so every level is one B2SR x bit
 * matrix product (OR.AND semiring).  d_levels: int32[n * k], vertex-major:
 * d_levels[v * k + s] = hops from h_srcs[s] to v, -1 if unreachable.  Needs a
 * square ROW-layout graph with 32x32 tiles.  No reference counterpart (the
 * reference runs one source per traversal, algorithm/bfs.cu:445). */
GBO_API int gbo_msbfs(const gbo_graph* g, const int* h_srcs, int k,
              int32_t* d_levels, int* h_depth, gbo_stream_t stream);
/* Multi-seed BFS: every vertex in h_seeds starts at level 0 of one frontier.
 * On a block-diagonal union of independent graphs (gbo_gen_er_batch) with one
 * seed per graph this is each graph's own BFS in one traversal. */
GBO_API int gbo_bfs_multi(const gbo_graph* g, const int* h_seeds, int nseeds,
                  int32_t* d_level, int* h_depth, gbo_stream_t stream);

/* Query server with continuous batching (no reference counterpart).  BFS
 * queries occupy columns of a multi-source BFS state (bfs_slots <= 1024,
 * rounded up to a multiple of 32) and join or leave at level boundaries;
 * PPR queries (1..64 weighted vertices, p = alpha P D^-1 p + (1-alpha) v,
 * stop at L1 change <= tol) occupy columns of a 32-wide fp32 matrix
 * (ppr_slots 0 or 32) and join or leave at iteration boundaries.  A worker
 * thread drives the GPU; submit/poll/wait are thread-safe.  Results: BFS
 * int32[n] levels (hops, -1 unreachable), PPR float[n].  A query's result
 * is the same whatever else is in flight.  Needs a square ROW-layout graph
 * with 32x32 tiles (and out-degrees for PPR).  A finished result waits in
 * a device buffer until wait/poll copies it to the caller, in any order;
 * while every buffer holds an uncollected result, finished queries keep
 * their slots until a client takes one. */
typedef struct gbo_server gbo_server;
typedef struct gbo_server_stats {
  long long rounds;          /* worker rounds (one BFS level or one PPR iteration) */
  long long bfs_completed, ppr_completed;
  long long kernel_launches;
  long long pending, in_flight;
  /* wall time per phase (ms, summed): the workers' BFS levels and PPR
   * iterations (kernels and the completion read-back) and retirements
   * (extraction into device result buffers), and the clients' result
   * copies (device to host, inside wait/poll) */
  double bfs_round_ms, ppr_round_ms, retire_ms, copy_ms;
  /* copy_ms split: waiting for the retirement kernel (with
   * gbo_server_wait_device: the whole device-side copy), the device-to-host
   * copy, and widening byte levels into the caller's int32 buffer */
  double copy_wait_ms, copy_d2h_ms, copy_widen_ms;
} gbo_server_stats;
GBO_API int gbo_server_create(const gbo_graph* g, int bfs_slots, int ppr_slots,
                      float alpha, float tol, int ppr_max_iter,
                      gbo_server** out);
/* Bound the admission queue: a submit that finds max_pending queries not
 * yet admitted returns GBO_ERR_FULL and queues nothing (0: unbounded, the
 * default).  The reference has no server; this is its request-overflow
 * policy. */
GBO_API int gbo_server_set_queue_limit(gbo_server* s, long long max_pending);
/* BFS admission batching: pending BFS queries enter the engine when at
 * least ceil(min_free_fraction * bfs_slots) slots are free, or when no
 * admitted query is still traversing.  0 admits into any free slot every
 * round; values below 1 trade a little latency for fewer rounds in which
 * freshly admitted sources keep every row of the graph open.  1 is batch
 * mode: queries enter only an idle engine whose results have all retired,
 * and each batch runs as one multi-source BFS (level 0 pushed from the
 * sources, finished columns retired, the narrowest frontier width that
 * holds the batch) into a level store of its own, then retires in one pass;
 * iterations then report the batch's depth.  Batch mode has the highest
 * capacity; clients that take results with gbo_server_wait_device on
 * streams of their own want more hardware queues than CUDA's default 8
 * (CUDA_DEVICE_MAX_CONNECTIONS=32 in the environment before CUDA starts),
 * or their copies queue behind the engine's traversal.  Default 0.5. */
GBO_API int gbo_server_set_admission(gbo_server* s, float min_free_fraction);
GBO_API int gbo_server_submit_bfs(gbo_server* s, int src, int64_t* ticket);
GBO_API int gbo_server_submit_ppr(gbo_server* s, const int* verts,
                          const float* weights, int count, int64_t* ticket);
/* GBO_OK and the result copied to h_out (may be NULL), or GBO_ERR_NOTREADY. */
GBO_API int gbo_server_poll(gbo_server* s, int64_t ticket, void* h_out,
                    double* latency_ms, int* iterations);
GBO_API int gbo_server_wait(gbo_server* s, int64_t ticket, void* h_out,
                    double* latency_ms, int* iterations, double timeout_s);
/* As gbo_server_wait for a BFS query, with the levels as one byte per
 * vertex (uint8[n]; 255 = unreachable): a quarter of the int32 result's
 * bytes over the host link and no widening.  When h_out is pinned
 * (gbo_host_alloc) the device copies straight into it.  A query deeper than
 * 254 levels keeps its result and returns GBO_ERR_OVERFLOW: collect it with
 * gbo_server_wait.  PPR tickets return GBO_ERR_INVALID. */
GBO_API int gbo_server_wait_u8(gbo_server* s, int64_t ticket, uint8_t* h_out,
                               double* latency_ms, int* iterations, double timeout_s);
/* As gbo_server_wait, but the result goes to the caller's device buffer
 * d_out (BFS int32[n] levels, PPR float[n]), for consumers that stay on the
 * GPU: no host copy.  The copy runs on `stream` (0: a high-priority stream
 * of the calling thread's own, so that it does not queue behind the
 * server's traversal kernels) and is complete when the call returns. */
GBO_API int gbo_server_wait_device(gbo_server* s, int64_t ticket, void* d_out,
                           double* latency_ms, int* iterations, double timeout_s,
                           gbo_stream_t stream);
GBO_API int gbo_server_get_stats(gbo_server* s, gbo_server_stats* stats);
GBO_API int gbo_server_destroy(gbo_server* s);

/* Personalized PageRank p = alpha * P D^-1 p + (1-alpha) v  (fp32) and its
 * adjoint: for loss L = dot(w, p), grad_v = (1-alpha) u with
 * u = alpha * D^-1 P^T u + w.  Iterate until the L1 change <= tol (forward:
 * v is a distribution) or <= tol * ||w||_1 (adjoint), or max_iter.  No
 * reference counterpart (built from A7). */
GBO_API int gbo_ppr_forward(const gbo_graph* g, const float* d_v, float alpha,
                    float tol, int max_iter, float* d_p, int* h_iters,
                    gbo_stream_t stream);
GBO_API int gbo_ppr_backward(const gbo_graph* g, const float* d_w, float alpha,
                     float tol, int max_iter, float* d_grad_v, int* h_iters,
                     gbo_stream_t stream);

/* Statistics of the last algorithm call on a graph (per-iteration device
 * time of the main BMV kernel, measured with CUDA events recorded inside the
 * captured iteration graph).  No reference counterpart (the reference's
 * GpuTimer brackets whole loops, algorithm/utility.cu:38). */
#define GBO_MAX_STEP_TIMES 256
typedef struct gbo_run_stats {
  int iterations;        /* iterations executed */
  int graph_replays;     /* CUDA graph launches (one host sync each) */
  long long kernel_launches;
  int nsteps;            /* entries of step_ms */
  float step_ms[GBO_MAX_STEP_TIMES];
} gbo_run_stats;
GBO_API int gbo_graph_last_run(const gbo_graph* g, gbo_run_stats* stats);

/* ------------------------------------------------ host CSR + I/O (A13) */
typedef struct gbo_csr {
  int nrows, ncols;
  int64_t nnz;
  int* rowptr; /* host, nrows+1 */
  int* colind; /* host, nnz     */
} gbo_csr;
enum { GBO_MTX_READMTX = 0, GBO_MTX_MMIO = 1 };
/* mode GBO_MTX_READMTX: readMtx + coo2csr semantics (readMtx.hpp:351-423,
 * 246-304): directed 0 = symmetrise iff the banner says symmetric, 1 = never,
 * 2 = always; self-loops and duplicates removed; rows sorted.
 * mode GBO_MTX_MMIO: mmio_data semantics (mmio_highlevel.h:139-309): banner
 * symmetry mirrors off-diagonal entries, self-loops and duplicates kept;
 * columns are sorted inside each row (order inside a row carries no meaning
 * for a binary matrix). */
GBO_API int gbo_read_mtx(const char* path, int mode, int directed, gbo_csr** out);
GBO_API int gbo_csr_free(gbo_csr* csr);
/* The same readers on the GPU: the entry lines are parsed in parallel and
 * the CSR is built in device memory -- identical to gbo_read_mtx's for
 * well-formed files (each line is parsed on its own).  d_rowptr (int32[nrows+1]) and d_colind (int32[nnz]) are
 * allocated here; free them with gbo_free.  gbo_graph_from_mtx packs the
 * parsed CSR straight into a graph (flags as gbo_graph_from_csr). */
GBO_API int gbo_read_mtx_device(const char* path, int mode, int directed,
                        int** d_rowptr, int** d_colind, int* nrows, int* ncols,
                        int64_t* nnz, gbo_stream_t stream);
GBO_API int gbo_graph_from_mtx(const char* path, int mode, int directed,
                       int tile_bits, int flags, gbo_stream_t stream,
                       gbo_graph** out);
/* CSC of a host CSR (readMtx.hpp:319-345), rows of the result sorted. */
GBO_API int gbo_csr_transpose(const gbo_csr* in, gbo_csr** out);
/* Keep entries with row >= col (tril_csr, bsrbmm/bsrbmm.cu:1416). */
GBO_API int gbo_csr_tril(const gbo_csr* in, gbo_csr** out);
/* Host CSR from an edge list: symmetrise (optional), drop self-loops
 * (optional), sort and deduplicate. */
GBO_API int gbo_csr_from_edges(const int* src, const int* dst, int64_t nedges,
                       int nvertices, int symmetrize, int drop_self_loops,
                       gbo_csr** out);

/* Seeded synthetic graphs (splitmix64 -> xoshiro256**; one stream per edge
 * draw, so the result does not depend on the thread count). */
GBO_API int gbo_gen_rmat(int scale, int edge_factor, double a, double b, double c,
                 uint64_t seed, gbo_csr** out);
GBO_API int gbo_gen_er(int n, double p, uint64_t seed, gbo_csr** out);
GBO_API int gbo_gen_er_avgdeg(int n, double avg_degree, uint64_t seed, gbo_csr** out);
GBO_API int gbo_gen_king_mesh(int side, gbo_csr** out);
/* count independent G(n, m) graphs as one block-diagonal CSR: n log-uniform in
 * [nmin, nmax], average degree avg_degree, graph i seeded with seed+1000+i;
 * offsets[count+1] receives each graph's first vertex. */
GBO_API int gbo_gen_er_batch(int count, int nmin, int nmax, double avg_degree,
                     uint64_t seed, gbo_csr** out, int* offsets);

/* ------------------------------------------------ host-side fault injection
 * For failure-path tests (the reference has no failure handling: its error
 * checks compile away, utility.cu:17-30).  Nothing here makes a GPU fault,
 * trap or hang; each knob changes a host-side decision (the last one a
 * launch argument).  Process-wide, off by default; n = 0 disarms.
 *   GBO_INJECT_HOST_ALLOC  (n >= 1) the n-th host CSR allocation from now on
 *       (readers, generators, CSR utilities) fails: the call returns
 *       GBO_ERR_NOMEM and leaves its output untouched;
 *   GBO_INJECT_REPLAY_CAP  (n >= 1) the iteration loops (BFS, SSSP,
 *       PageRank, PPR, CC) replay their captured iterations at most n times
 *       and return GBO_ERR_TIMEOUT when the device has not finished by then;
 *   GBO_INJECT_SERVER_HOLD (n = 1) server workers admit no new query:
 *       submissions stay pending (queries already in flight finish);
 *   GBO_INJECT_BARRIER_SKIP (n >= 1) the next cooperative BFS launch (one
 *       shot) is told that block n - 1 leaves before the first grid barrier
 *       and that the barrier gives up after 100 ms instead of 5 s: the other
 *       blocks' bounded wait runs out, every block leaves, and the
 *       synchronous call returns GBO_ERR_TIMEOUT with the context usable. */
enum { GBO_INJECT_HOST_ALLOC = 1, GBO_INJECT_REPLAY_CAP = 2, GBO_INJECT_SERVER_HOLD = 3,
       GBO_INJECT_BARRIER_SKIP = 4 };
GBO_API int gbo_debug_inject(int what, long long n);

#ifdef __cplusplus
}
#endif
#endif /* GBO_H_ */
