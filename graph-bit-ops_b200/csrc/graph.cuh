// The device-resident B2SR graph behind the opaque gbo_graph handle, and the
// warp work-item schedule that balances power-law block rows.
#pragma once

#include "common.cuh"

// One warp-group work item: tiles [t0, t1) of block row `row`.  A block row
// with more tiles than the chunk size is split into several items; those
// write partial results into scratch `slot` and a reduce kernel combines
// them in slot order (deterministic, also for floating point).
struct __align__(16) gbo_item {
  int row, t0, t1, slot;  // slot = -1: the item covers its whole row
};
// A split block row: its partial results live in slots [slot0, slot0+n).
struct __align__(16) gbo_split {
  int row, slot0, nslots, pad;
};

struct gbo_graph {
  int nrows = 0, ncols = 0, b = 0, layout = GBO_LAYOUT_ROW;
  int nbr = 0, nbc = 0;
  long long nblk = 0, nnz = -1;
  int* rowptr = nullptr;   // nbr+1
  int* colind = nullptr;   // nblk
  void* val = nullptr;     // nblk*b words
  int* outdeg = nullptr;   // ncols (column counts of P), may be null
  float* invdeg = nullptr; // 1/outdeg (0 where outdeg == 0), may be null
  bool owns_b2sr = true;
  bool symmetric = false;  // caller asserts P == P^T (enables push BFS steps)
  int bfs_push_thr = -1;   // push below this frontier size (-1: nrows / 64)
  int bfs_loop = 0;        // GBO_BFS_LOOP_* (gbo_graph_set_bfs_loop)
  int bfs_coop_blocks = 0; // cooperative BFS grid (0: sized by the graph)
  int* perm = nullptr;     // GBO_FLAG_DEGREE_ORDER: new label of every input vertex
  int* tile_row = nullptr; // block row of every tile (triangle counting)
  unsigned* rowmask = nullptr;  // b = 32 ROW: non-empty row words of every tile
  unsigned* rowword = nullptr;  // b = 32 ROW: the non-empty row words, packed in tile order
  long long* item_wbase = nullptr;  // index in rowword of every work item's first word
  long long nrowword = 0;
  // b = 32 ROW, built on first BFS use (build_rws): every row's non-empty
  // row words with their block columns in ascending block-column order; the
  // first kRwsHead entries of the 32 rows of a block row entry-major, the
  // rest in per-row tails
  uint2* rws_head = nullptr;       // nbr * kRwsHead * 32 entries {block column, row word}
  uint2* rws_tail = nullptr;       // entries past the head, row after row
  long long* rws_tail_ptr = nullptr;  // nbr * 32 + 1 offsets into rws_tail
  // rows whose tails are longer than kRwsLongTail, cut into chunks of at most
  // kRwsChunk tail entries, for kernels that must read whole rows (PageRank):
  // long row q owns chunks [rws_long_chunk0[q], rws_long_chunk0[q + 1])
  int rws_nlong = 0;
  long long rws_nchunk = 0;
  long long rws_ntail = 0;  // entries in rws_tail
  int* rws_long_row = nullptr;         // rws_nlong rows
  long long* rws_long_chunk0 = nullptr;  // rws_nlong + 1
  int* rws_chunk_row = nullptr;        // row of every chunk
  long long* rws_chunk_beg = nullptr;  // tail entries [beg, end) of every chunk
  long long* rws_chunk_end = nullptr;
  unsigned* rws_longbits = nullptr;    // nbr words: bit 31 - r set when row 32R + r is long
  int last_run_ms = 0;     // 1: the last traversal was a multi-source BFS
  bool tc_mma = false;     // GBO_FLAG_TC_MMA: dense 32x32 mask tiles on the 1-bit MMA
  bool owns_outdeg = true;
  // balanced schedule
  int chunk = 0;
  int nitems = 0;
  gbo_item* items = nullptr;
  int nsplit = 0;
  gbo_split* splits = nullptr;
  int nslots = 0;
  // per-handle workspace for BMV split partials (grown on demand)
  void* ws = nullptr;
  size_t ws_bytes = 0;
  long long device_bytes = 0;
  // device state and captured CUDA graphs of the iteration loops
  struct AlgoState* algo = nullptr;
  void* ms = nullptr;  // multi-source BFS state
};

namespace gbo {

// Chunk (tiles per work item) for a tile width.
inline int chunk_for(int b) {
  switch (b) {
    case 4: return 2048;
    case 8: return 1024;
    case 16: return 512;
    case 32: return 256;
    default: return 128;
  }
}

// Work items processed per warp: 32/b groups for b <= 32, one for b = 64.
inline int groups_per_warp(int b) { return b >= 32 ? 1 : 32 / b; }

// Build items/splits for g (rowptr must be set).  Allocates g->items/splits.
int build_schedule(gbo_graph* g, cudaStream_t stream);

// Row-occupancy words of b = 32 ROW tiles -> g->rowmask (no-op otherwise).
int build_rowmask(gbo_graph* g, cudaStream_t stream);
// Packed non-empty row words -> g->rowword, g->item_wbase (needs rowmask and
// the schedule; no-op without them).
int build_rowwords(gbo_graph* g, cudaStream_t stream);

// Entries per row held entry-major in the row-word slices' head, and the
// block column that marks a missing entry.
constexpr int kRwsHead = 8;
constexpr unsigned kRwsNone = 0xffffffffu;
// Tails longer than this are walked by a whole warp (BFS) or cut into
// chunks of kRwsChunk entries spread over warps (PageRank).
constexpr int kRwsLongTail = 64;
constexpr int kRwsChunk = 512;
// Row-word slices of a b = 32 ROW graph -> g->rws_* (no-op for other graphs
// or when built).  Needs g->rowmask.
int build_rws(gbo_graph* g, cudaStream_t stream);

// Ensure g->ws has at least `bytes` (contents undefined).
int ensure_workspace(gbo_graph* g, size_t bytes, cudaStream_t stream);

// Pack CSR (device pointers) into B2SR owned by g.  Sets nblk, rowptr, colind,
// val.  Synchronises the stream once (to size the tile arrays).
// Per block row, the rows of P that have an entry (bit b-1-r of word R),
// computed once per graph on `s` and owned by the graph's algorithm state.
int live_rows(gbo_graph* g, cudaStream_t s, const void** out);
int count_tiles(const int* d_rowptr, const int* d_colind, int nrows, int ncols, long long nnz, int b,
                long long* nblk, cudaStream_t s);
int pack_into(gbo_graph* g, const int* d_rowptr, const int* d_colind, int nrows, int ncols,
              long long nnz, int b, int layout, cudaStream_t stream);

// Column counts of a CSR (device) -> g->outdeg, g->invdeg.
int compute_outdeg_from_cols(gbo_graph* g, const int* d_colind, long long nnz, int ncols,
                             cudaStream_t stream);
int compute_outdeg_from_rowptr(gbo_graph* g, const int* d_rowptr, int nrows, cudaStream_t stream);
// Out-degrees given on the host (n ints) -> g->outdeg, g->invdeg.
int upload_outdeg(gbo_graph* g, const int* h_deg, int n, cudaStream_t stream);
// inv[i] = 1/deg[i] (0 where deg is 0).
void launch_invdeg(const int* d_deg, int n, float* d_inv, cudaStream_t stream);
// Release the algorithm state of g (called by gbo_graph_free).
void free_algo_state(gbo_graph* g);
void free_ms_state(gbo_graph* g);
// Statistics of the last multi-source BFS (per-level times of its step kernel).
int ms_last_run(const gbo_graph* g, gbo_run_stats* stats);

}  // namespace gbo
