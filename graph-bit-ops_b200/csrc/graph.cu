// Graph handle construction and the C ABI of the BMV primitives.
#include <algorithm>
#include <cmath>
#include <vector>

#include "bmv.cuh"

namespace gbo {

namespace {

// Device copy of a CSR given by host or device pointers, optionally filtered
// to the lower triangle (row >= col) -- tril_csr (bsrbmm/bsrbmm.cu:1416).
__global__ void k_tril_count(const int* __restrict__ rowptr, const int* __restrict__ colind,
                             int nrows, int* __restrict__ cnt) {
  const long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31;
  if (row >= nrows) return;
  int a = rowptr[row], e = rowptr[row + 1];
  int c = 0;
  for (int p = a + (int)lane; p < e; p += 32) c += colind[p] <= row;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (lane == 0) cnt[row] = c;
}

__global__ void k_tril_fill(const int* __restrict__ rowptr, const int* __restrict__ colind,
                            int nrows, const int* __restrict__ newptr, int* __restrict__ newcol) {
  const long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31;
  if (row >= nrows) return;
  int a = rowptr[row], e = rowptr[row + 1];
  int out = newptr[row];
  for (int base = a; base < e; base += 32) {
    int p = base + (int)lane;
    bool keep = p < e && colind[p] <= row;
    unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (keep) newcol[out + __popc(bal & ((1u << lane) - 1u))] = colind[p];
    out += __popc(bal);
  }
}

struct DevCsr {
  int* rowptr = nullptr;
  int* colind = nullptr;
  long long nnz = 0;
  bool owned = false;
  void release() {
    if (owned) {
      cudaFree(rowptr);
      cudaFree(colind);
    }
    rowptr = colind = nullptr;
    owned = false;
  }
};

int upload_csr(const int* rowptr, const int* colind, int nrows, long long nnz, bool device,
               cudaStream_t s, DevCsr* out) {
  if (device) {
    out->rowptr = const_cast<int*>(rowptr);
    out->colind = const_cast<int*>(colind);
    out->nnz = nnz;
    out->owned = false;
    return GBO_OK;
  }
  GBO_CUDA_TRY(cudaMalloc(&out->rowptr, sizeof(int) * ((size_t)nrows + 1)));
  GBO_CUDA_TRY(cudaMalloc(&out->colind, sizeof(int) * (size_t)(nnz > 0 ? nnz : 1)));
  out->owned = true;
  out->nnz = nnz;
  GBO_CUDA_TRY(cudaMemcpyAsync(out->rowptr, rowptr, sizeof(int) * ((size_t)nrows + 1),
                               cudaMemcpyHostToDevice, s));
  if (nnz > 0)
    GBO_CUDA_TRY(cudaMemcpyAsync(out->colind, colind, sizeof(int) * (size_t)nnz,
                                 cudaMemcpyHostToDevice, s));
  return GBO_OK;
}

int tril_device(const DevCsr& in, int nrows, cudaStream_t s, DevCsr* out) {
  int* cnt = nullptr;
  GBO_CUDA_TRY(pool_malloc_async(&cnt, sizeof(int) * ((size_t)nrows + 1), s));
  GBO_CUDA_TRY(cudaMalloc(&out->rowptr, sizeof(int) * ((size_t)nrows + 1)));
  out->owned = true;
  long long* tot = nullptr;
  GBO_CUDA_TRY(pool_malloc_async(&tot, sizeof(long long), s));
  if (nrows > 0) k_tril_count<<<blocks_for_warps(nrows, 8), 256, 0, s>>>(in.rowptr, in.colind, nrows, cnt);
  GBO_TRY(exclusive_scan_i32(cnt, out->rowptr, nrows, tot, s));
  long long h = 0;
  GBO_CUDA_TRY(cudaMemcpyAsync(&h, tot, sizeof(long long), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  out->nnz = h;
  GBO_CUDA_TRY(cudaMalloc(&out->colind, sizeof(int) * (size_t)(h > 0 ? h : 1)));
  if (nrows > 0)
    k_tril_fill<<<blocks_for_warps(nrows, 8), 256, 0, s>>>(in.rowptr, in.colind, nrows, out->rowptr,
                                                          out->colind);
  GBO_CUDA_TRY(cudaGetLastError());
  cudaFreeAsync(cnt, s);
  cudaFreeAsync(tot, s);
  return GBO_OK;
}

void destroy(gbo_graph* g) {
  if (!g) return;
  if (g->owns_b2sr) {
    cudaFree(g->rowptr);
    cudaFree(g->colind);
    cudaFree(g->val);
  }
  if (g->owns_outdeg) cudaFree(g->outdeg);
  cudaFree(g->perm);
  cudaFree(g->tile_row);
  cudaFree(g->rowmask);
  cudaFree(g->rowword);
  cudaFree(g->item_wbase);
  cudaFree(g->rws_head);
  cudaFree(g->rws_tail);
  cudaFree(g->rws_tail_ptr);
  cudaFree(g->rws_long_row);
  cudaFree(g->rws_long_chunk0);
  cudaFree(g->rws_chunk_row);
  cudaFree(g->rws_chunk_beg);
  cudaFree(g->rws_chunk_end);
  cudaFree(g->rws_longbits);
  cudaFree(g->invdeg);
  cudaFree(g->items);
  cudaFree(g->splits);
  cudaFree(g->ws);
  free_algo_state(g);
  free_ms_state(g);
  delete g;
}

}  // namespace

// Host CSR transpose used when GBO_FLAG_TRANSPOSE is given with host pointers.
int host_transpose(const int* rowptr, const int* colind, int nrows, int ncols, long long nnz,
                   std::vector<int>* tptr, std::vector<int>* tcol);
// Host relabelling by descending degree (GBO_FLAG_DEGREE_ORDER).
int host_degree_relabel(const int* rowptr, const int* colind, int n, long long nnz,
                        std::vector<int>* new_of_old, std::vector<int>* nptr, std::vector<int>* ncol);

}  // namespace gbo

using namespace gbo;

extern "C" int gbo_graph_from_csr(const int* rowptr, const int* colind, int nrows, int ncols,
                                  int nnz, int tile_bits, int flags, gbo_stream_t stream,
                                  gbo_graph** out) {
  clear_error();
  if (!out) return fail(GBO_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (!valid_tile_bits(tile_bits)) return fail(GBO_ERR_INVALID, "tile_bits must be 4, 8, 16, 32 or 64");
  if (nrows < 0 || ncols < 0 || nnz < 0 || !rowptr || (nnz > 0 && !colind))
    return fail(GBO_ERR_INVALID, "gbo_graph_from_csr: bad CSR argument");
  const bool device = flags & GBO_FLAG_DEVICE_PTRS;
  const bool transpose = flags & GBO_FLAG_TRANSPOSE;
  const bool lower = flags & GBO_FLAG_LOWER;
  const int layout = (flags & GBO_FLAG_LAYOUT_COL) ? GBO_LAYOUT_COL : GBO_LAYOUT_ROW;
  if (lower && nrows != ncols) return fail(GBO_ERR_INVALID, "GBO_FLAG_LOWER needs a square matrix");
  cudaStream_t s = as_stream(stream);

  // Transpose (CSC) on the host side of the boundary when given host arrays;
  // device arrays are copied back first.  The packer needs sorted rows, and
  // the host transpose emits them in ascending order like readMtx's csr2csc.
  std::vector<int> tptr, tcol, hptr, hcol;
  const int* src_ptr = rowptr;
  const int* src_col = colind;
  int prow = nrows, pcol = ncols;
  bool src_device = device;
  if (transpose) {
    if (device) {
      hptr.resize((size_t)nrows + 1);
      hcol.resize((size_t)nnz);
      GBO_CUDA_TRY(cudaMemcpyAsync(hptr.data(), rowptr, sizeof(int) * hptr.size(), cudaMemcpyDeviceToHost, s));
      if (nnz) GBO_CUDA_TRY(cudaMemcpyAsync(hcol.data(), colind, sizeof(int) * hcol.size(), cudaMemcpyDeviceToHost, s));
      GBO_CUDA_TRY(cudaStreamSynchronize(s));
      src_ptr = hptr.data();
      src_col = hcol.data();
    }
    GBO_TRY(host_transpose(src_ptr, src_col, nrows, ncols, nnz, &tptr, &tcol));
    src_ptr = tptr.data();
    src_col = tcol.data();
    prow = ncols;
    pcol = nrows;
    src_device = false;
  }
  // Relabel by descending degree: the packed matrix is P' = Q P Q^T.  Row
  // lengths of the lower triangle are then bounded by the number of
  // higher-degree neighbours, which keeps hub rows short for TC.
  std::vector<int> perm, rptr, rcol;
  if (flags & GBO_FLAG_DEGREE_ORDER) {
    if (prow != pcol) return fail(GBO_ERR_INVALID, "GBO_FLAG_DEGREE_ORDER needs a square matrix");
    if (transpose) return fail(GBO_ERR_UNSUPPORTED, "GBO_FLAG_DEGREE_ORDER does not combine with GBO_FLAG_TRANSPOSE");
    if (src_device) {
      hptr.resize((size_t)prow + 1);
      hcol.resize((size_t)nnz);
      GBO_CUDA_TRY(cudaMemcpyAsync(hptr.data(), src_ptr, sizeof(int) * hptr.size(), cudaMemcpyDeviceToHost, s));
      if (nnz) GBO_CUDA_TRY(cudaMemcpyAsync(hcol.data(), src_col, sizeof(int) * hcol.size(), cudaMemcpyDeviceToHost, s));
      GBO_CUDA_TRY(cudaStreamSynchronize(s));
      src_ptr = hptr.data();
      src_col = hcol.data();
      src_device = false;
    }
    GBO_TRY(host_degree_relabel(src_ptr, src_col, prow, nnz, &perm, &rptr, &rcol));
    src_ptr = rptr.data();
    src_col = rcol.data();
  }

  gbo_graph* g = new gbo_graph();
  g->symmetric = (flags & GBO_FLAG_SYMMETRIC) && !lower && nrows == ncols;
  g->tc_mma = (flags & GBO_FLAG_TC_MMA) != 0;
  if (!perm.empty()) {
    if (cudaMalloc(&g->perm, sizeof(int) * perm.size()) != cudaSuccess ||
        cudaMemcpy(g->perm, perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
      destroy(g);
      return fail(GBO_ERR_NOMEM, "permutation upload");
    }
    g->device_bytes += 4LL * (long long)perm.size();
  }
  DevCsr csr, low;
  int st = upload_csr(src_ptr, src_col, prow, nnz, src_device, s, &csr);
  const DevCsr* use = &csr;
  if (st == GBO_OK && lower) {
    st = tril_device(csr, prow, s, &low);
    use = &low;
  }
  if (st == GBO_OK) st = pack_into(g, use->rowptr, use->colind, prow, pcol, use->nnz, tile_bits, layout, s);
  // out-degree of the graph P pulls over: column counts of P.  With
  // GBO_FLAG_TRANSPOSE these are the row lengths of the given CSR
  // (the reference reads csrRowPtr deltas, algorithm/bsrbmv.cu:1277).
  if (st == GBO_OK) {
    if (transpose) {
      const int* hp = device ? hptr.data() : rowptr;
      std::vector<int> deg((size_t)nrows);
      for (int i = 0; i < nrows; ++i) deg[i] = hp[i + 1] - hp[i];
      st = upload_outdeg(g, deg.data(), nrows, s);
      if (st == GBO_OK) st = cudaStreamSynchronize(s) == cudaSuccess ? GBO_OK : fail(GBO_ERR_CUDA, "sync");
    } else {
      st = compute_outdeg_from_cols(g, use->colind, use->nnz, pcol, s);
    }
  }
  if (st == GBO_OK) st = build_schedule(g, s);
  if (st == GBO_OK) st = build_rowmask(g, s);
  if (st == GBO_OK) st = build_rowwords(g, s);
  if (st == GBO_OK) st = ensure_workspace(g, bmv_scratch_bytes(g), s);
  if (st == GBO_OK) st = cudaStreamSynchronize(s) == cudaSuccess ? GBO_OK : fail(GBO_ERR_CUDA, "graph build sync");
  low.release();
  csr.release();
  if (st != GBO_OK) {
    destroy(g);
    return st;
  }
  *out = g;
  return GBO_OK;
}

extern "C" int gbo_graph_wrap_b2sr(int nrows, int ncols, int tile_bits, int layout, int nblocks,
                                   const int* d_bsrRowPtr, const int* d_bsrColInd,
                                   const void* d_bsrVal, const int* d_outdeg, gbo_stream_t stream,
                                   gbo_graph** out) {
  clear_error();
  if (!out) return fail(GBO_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (!valid_tile_bits(tile_bits)) return fail(GBO_ERR_INVALID, "tile_bits must be 4, 8, 16, 32 or 64");
  if (nrows < 0 || ncols < 0 || nblocks < 0 || !d_bsrRowPtr || (nblocks > 0 && (!d_bsrColInd || !d_bsrVal)))
    return fail(GBO_ERR_INVALID, "gbo_graph_wrap_b2sr: bad argument");
  if (layout != GBO_LAYOUT_ROW && layout != GBO_LAYOUT_COL) return fail(GBO_ERR_INVALID, "bad layout");
  cudaStream_t s = as_stream(stream);
  gbo_graph* g = new gbo_graph();
  g->nrows = nrows;
  g->ncols = ncols;
  g->b = tile_bits;
  g->layout = layout;
  g->nbr = (nrows + tile_bits - 1) / tile_bits;
  g->nbc = (ncols + tile_bits - 1) / tile_bits;
  g->nblk = nblocks;
  g->rowptr = const_cast<int*>(d_bsrRowPtr);
  g->colind = const_cast<int*>(d_bsrColInd);
  g->val = const_cast<void*>(d_bsrVal);
  g->owns_b2sr = false;
  g->owns_outdeg = false;
  int st = GBO_OK;
  if (d_outdeg) {
    g->outdeg = const_cast<int*>(d_outdeg);
    if (cudaMalloc(&g->invdeg, sizeof(float) * (size_t)(ncols > 0 ? ncols : 1)) != cudaSuccess)
      st = fail(GBO_ERR_NOMEM, "invdeg");
    if (st == GBO_OK) launch_invdeg(d_outdeg, ncols, g->invdeg, s);
  }
  if (st == GBO_OK) st = build_schedule(g, s);
  if (st == GBO_OK) st = build_rowmask(g, s);
  if (st == GBO_OK) st = build_rowwords(g, s);
  if (st == GBO_OK) st = ensure_workspace(g, bmv_scratch_bytes(g), s);
  if (st == GBO_OK) st = cudaStreamSynchronize(s) == cudaSuccess ? GBO_OK : fail(GBO_ERR_CUDA, "wrap sync");
  if (st != GBO_OK) {
    destroy(g);
    return st;
  }
  *out = g;
  return GBO_OK;
}

extern "C" int gbo_graph_free(gbo_graph* g) {
  clear_error();
  destroy(g);
  return GBO_OK;
}

extern "C" int gbo_graph_get_info(const gbo_graph* g, gbo_graph_info* info) {
  clear_error();
  if (!g || !info) return fail(GBO_ERR_INVALID, "NULL argument");
  info->nrows = g->nrows;
  info->ncols = g->ncols;
  info->tile_bits = g->b;
  info->layout = g->layout;
  info->nblockrows = g->nbr;
  info->nblockcols = g->nbc;
  info->nblocks = g->nblk;
  info->nnz = g->nnz;
  info->b2sr_bytes = 4LL * (g->nbr + 1) + 4LL * g->nblk + g->nblk * (long long)g->b * word_bytes(g->b);
  info->device_bytes = g->device_bytes;
  info->nsplit_rows = g->nsplit;
  info->nitems = g->nitems;
  return GBO_OK;
}

extern "C" int gbo_graph_b2sr(const gbo_graph* g, const int** r, const int** c, const void** v) {
  clear_error();
  if (!g) return fail(GBO_ERR_INVALID, "NULL graph");
  if (r) *r = g->rowptr;
  if (c) *c = g->colind;
  if (v) *v = g->val;
  return GBO_OK;
}

extern "C" int gbo_graph_outdeg(const gbo_graph* g, const int** d) {
  clear_error();
  if (!g || !d) return fail(GBO_ERR_INVALID, "NULL argument");
  *d = g->outdeg;
  return GBO_OK;
}

extern "C" int gbo_graph_permutation(const gbo_graph* g, const int** d_new_of_old) {
  clear_error();
  if (!g || !d_new_of_old) return fail(GBO_ERR_INVALID, "NULL argument");
  *d_new_of_old = g->perm;
  return GBO_OK;
}

extern "C" int gbo_graph_set_bfs_direction(gbo_graph* g, int symmetric, int push_threshold) {
  clear_error();
  if (!g) return fail(GBO_ERR_INVALID, "NULL graph");
  if (push_threshold < -1) return fail(GBO_ERR_INVALID, "push_threshold must be >= -1");
  if (symmetric && g->nrows != g->ncols) return fail(GBO_ERR_UNSUPPORTED, "push steps need a square graph");
  g->symmetric = symmetric != 0;
  g->bfs_push_thr = push_threshold;
  return GBO_OK;
}

extern "C" int gbo_graph_set_bfs_loop(gbo_graph* g, int loop, int coop_blocks) {
  clear_error();
  if (!g) return fail(GBO_ERR_INVALID, "NULL graph");
  if (loop < GBO_BFS_LOOP_AUTO || loop > GBO_BFS_LOOP_COOP) return fail(GBO_ERR_INVALID, "unknown BFS loop");
  if (coop_blocks < 0) return fail(GBO_ERR_INVALID, "coop_blocks must be >= 0");
  if (loop == GBO_BFS_LOOP_COOP && (g->b != 32 || g->layout != GBO_LAYOUT_ROW))
    return fail(GBO_ERR_UNSUPPORTED, "the cooperative BFS loop needs a b = 32 ROW graph");
  g->bfs_loop = loop;
  g->bfs_coop_blocks = coop_blocks;
  return GBO_OK;
}

// ------------------------------------------------------------ BMV C ABI
static int check_graph(const gbo_graph* g) {
  if (!g) return fail(GBO_ERR_INVALID, "graph is NULL");
  return GBO_OK;
}

extern "C" int gbo_bmv_count(const gbo_graph* g, const void* d_x_bits, void* d_y, int out_type,
                             int accumulate, gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_graph(g));
  if ((g->nrows > 0 && !d_y) || (g->nblk > 0 && !d_x_bits)) return fail(GBO_ERR_INVALID, "NULL vector");
  if (out_type != GBO_OUT_I32 && out_type != GBO_OUT_F32) return fail(GBO_ERR_INVALID, "bad out_type");
  if (g->layout != GBO_LAYOUT_ROW) return fail(GBO_ERR_UNSUPPORTED, "BMV needs the ROW tile layout");
  return bmv_count(g, d_x_bits, d_y, out_type, accumulate, g->ws, as_stream(stream));
}

extern "C" int gbo_bmv_masked(const gbo_graph* g, const void* d_x_bits, const void* d_mask_bits,
                              void* d_out_bits, gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_graph(g));
  if ((g->nbr > 0 && !d_out_bits) || (g->nblk > 0 && !d_x_bits)) return fail(GBO_ERR_INVALID, "NULL vector");
  if (g->layout != GBO_LAYOUT_ROW) return fail(GBO_ERR_UNSUPPORTED, "BMV needs the ROW tile layout");
  return bmv_masked(g, d_x_bits, d_mask_bits, d_out_bits, g->ws, as_stream(stream));
}

extern "C" int gbo_bmv_minplus(const gbo_graph* g, const uint32_t* d_x, uint32_t* d_y,
                               gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_graph(g));
  if (g->nrows > 0 && (!d_x || !d_y)) return fail(GBO_ERR_INVALID, "NULL vector");
  if (g->layout != GBO_LAYOUT_ROW) return fail(GBO_ERR_UNSUPPORTED, "BMV needs the ROW tile layout");
  if (d_x == d_y) return fail(GBO_ERR_INVALID, "x and y must not alias");
  if (g->nrows > g->ncols) return fail(GBO_ERR_INVALID, "min-plus over (P + I) needs nrows <= ncols");
  return bmv_minplus(g, d_x, d_y, g->ws, as_stream(stream));
}

extern "C" int gbo_bmv_float(const gbo_graph* g, const float* d_x, float* d_y, float alpha,
                             const float* d_scale, float add, gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_graph(g));
  if (g->nrows > 0 && (!d_x || !d_y)) return fail(GBO_ERR_INVALID, "NULL vector");
  if (g->layout != GBO_LAYOUT_ROW) return fail(GBO_ERR_UNSUPPORTED, "BMV needs the ROW tile layout");
  if (d_x == d_y) return fail(GBO_ERR_INVALID, "x and y must not alias");
  return bmv_float(g, d_x, d_y, alpha, d_scale, add, g->ws, as_stream(stream));
}

extern "C" int gbo_bmv_float_degptr(const gbo_graph* g, const float* d_x, float* d_y, float alpha,
                                    const int* d_csrRowPtr, gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_graph(g));
  if (g->nrows > 0 && (!d_x || !d_y || !d_csrRowPtr)) return fail(GBO_ERR_INVALID, "NULL vector");
  if (g->layout != GBO_LAYOUT_ROW) return fail(GBO_ERR_UNSUPPORTED, "BMV needs the ROW tile layout");
  if (d_x == d_y) return fail(GBO_ERR_INVALID, "x and y must not alias");
  return bmv_float(g, d_x, d_y, alpha, nullptr, 0.f, g->ws, as_stream(stream), d_csrRowPtr);
}

extern "C" int gbo_bmv_minselect(const gbo_graph* g, const int32_t* d_x, int32_t* d_y,
                                 gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_graph(g));
  if (g->nrows > 0 && (!d_x || !d_y)) return fail(GBO_ERR_INVALID, "NULL vector");
  if (g->layout != GBO_LAYOUT_ROW) return fail(GBO_ERR_UNSUPPORTED, "BMV needs the ROW tile layout");
  if (d_x == d_y) return fail(GBO_ERR_INVALID, "x and y must not alias");
  return bmv_minselect(g, d_x, d_y, g->ws, as_stream(stream));
}

extern "C" int gbo_bmv_float_transposed(const gbo_graph* g, const float* d_x, float* d_y,
                                        float alpha, const float* d_scale, float add,
                                        gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_graph(g));
  if (g->nrows > 0 && (!d_x || !d_y)) return fail(GBO_ERR_INVALID, "NULL vector");
  if (g->layout != GBO_LAYOUT_ROW) return fail(GBO_ERR_UNSUPPORTED, "BMV needs the ROW tile layout");
  if ((const void*)d_x == (const void*)d_y) return fail(GBO_ERR_INVALID, "x and y must not alias");
  return bmv_float_transposed(g, d_x, d_y, alpha, d_scale, add, as_stream(stream));
}

// ------------------------------------------------------------ tile tuner
// Pick the tile width for a matrix and an operation.  MODEL ranks the widths
// by the algorithmic bytes of one sweep over the packing (tile words +
// column indices + block-row offsets), from the packer's count pass alone;
// TIMED packs the matrix at every width and times the operation with CUDA
// events (one warm-up, three timed runs), keeping the fastest.
// Row words of a 32x32 packing: distinct (row, column / 32) pairs of a
// column-sorted CSR (a thread per row; one atomic add per block).
__global__ void k_count_row_words32(const int* __restrict__ rowptr, const int* __restrict__ colind, int nrows,
                                    unsigned long long* __restrict__ out) {
  unsigned long long c = 0;
  for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < nrows;
       u += (long long)gridDim.x * blockDim.x) {
    int prev = -1;
    for (int p = rowptr[u]; p < rowptr[u + 1]; ++p) {
      const int w = colind[p] >> 5;
      c += w != prev;
      prev = w;
    }
  }
  __shared__ unsigned long long sh;
  if (threadIdx.x == 0) sh = 0;
  __syncthreads();
  if (c) atomicAdd(&sh, c);
  __syncthreads();
  if (threadIdx.x == 0 && sh) atomicAdd(out, sh);
}

extern "C" int gbo_tune_tile_width(const int* rowptr, const int* colind, int nrows, int ncols,
                                   int nnz, int flags, int op, int mode, gbo_stream_t stream,
                                   int* best_bits, double* cost) {
  clear_error();
  static const int kWidths[5] = {4, 8, 16, 32, 64};
  if (!best_bits) return fail(GBO_ERR_INVALID, "best_bits is NULL");
  if (op != GBO_TUNE_BMV && op != GBO_TUNE_BFS && op != GBO_TUNE_TC) return fail(GBO_ERR_INVALID, "bad op");
  if (mode != GBO_TUNE_MODEL && mode != GBO_TUNE_TIMED) return fail(GBO_ERR_INVALID, "bad mode");
  if (nrows < 0 || ncols < 0 || nnz < 0 || !rowptr || (nnz > 0 && !colind))
    return fail(GBO_ERR_INVALID, "gbo_tune_tile_width: bad CSR argument");
  if (op == GBO_TUNE_TC) flags |= GBO_FLAG_LOWER;
  if ((flags & GBO_FLAG_LOWER) && nrows != ncols) return fail(GBO_ERR_INVALID, "TC needs a square matrix");
  cudaStream_t s = as_stream(stream);
  double c[5];
  if (mode == GBO_TUNE_MODEL) {
    // tile counts of P and P^T are equal, so the transpose is never built
    DevCsr csr, low;
    int st = upload_csr(rowptr, colind, nrows, nnz, flags & GBO_FLAG_DEVICE_PTRS, s, &csr);
    const DevCsr* use = &csr;
    if (st == GBO_OK && (flags & GBO_FLAG_LOWER)) {
      st = tril_device(csr, nrows, s, &low);
      use = &low;
    }
    for (int k = 0; k < 5 && st == GBO_OK; ++k) {
      const int b = kWidths[k];
      long long nblk = 0;
      st = count_tiles(use->rowptr, use->colind, nrows, ncols, use->nnz, b, &nblk, s);
      if (st == GBO_OK) {
        const double wb = b >= 8 ? b / 8 : 1;
        c[k] = (double)nblk * (b * wb + 4.0) + 4.0 * ((nrows + b - 1) / b + 1);
        if (op == GBO_TUNE_BFS && b == 32 && !(flags & GBO_FLAG_LAYOUT_COL) && nrows > 0) {
          // 32x32 ROW BFS walks row-word slices: 8 bytes per non-empty row
          // word and 8 per row of tail offsets in one pass (its pull steps
          // stop at a row's first frontier neighbour, so a BFS reads less)
          unsigned long long* d = nullptr;
          unsigned long long rw = 0;
          if (pool_malloc_async(&d, sizeof(rw), s) != cudaSuccess || cudaMemsetAsync(d, 0, sizeof(rw), s) != cudaSuccess) {
            st = fail(GBO_ERR_NOMEM, "tuner counter");
          } else {
            const int grid = (int)std::min<long long>(((long long)nrows + 255) / 256, 4096);
            k_count_row_words32<<<grid, 256, 0, s>>>(use->rowptr, use->colind, nrows, d);
            if (cudaMemcpyAsync(&rw, d, sizeof(rw), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess)
              st = fail(GBO_ERR_CUDA, "tuner row-word count");
            cudaFreeAsync(d, s);
            if (st == GBO_OK) c[k] = 8.0 * (double)rw + 8.0 * ((double)nrows + 1.0);
          }
        }
      } else if (st == GBO_ERR_OVERFLOW) {
        c[k] = INFINITY;
        st = GBO_OK;
        clear_error();
      }
    }
    if (st == GBO_OK) st = cudaStreamSynchronize(s) == cudaSuccess ? GBO_OK : fail(GBO_ERR_CUDA, "tuner sync");
    low.release();
    csr.release();
    if (st != GBO_OK) return st;
  } else {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    GBO_CUDA_TRY(cudaEventCreate(&e0));
    GBO_CUDA_TRY(cudaEventCreate(&e1));
    int st = GBO_OK;
    for (int k = 0; k < 5 && st == GBO_OK; ++k) {
      const int b = kWidths[k];
      gbo_graph* g = nullptr;
      st = gbo_graph_from_csr(rowptr, colind, nrows, ncols, nnz, b, flags, stream, &g);
      if (st == GBO_ERR_OVERFLOW) {  // too many tiles at this width
        c[k] = INFINITY;
        st = GBO_OK;
        clear_error();
        continue;
      }
      if (st != GBO_OK) break;
      void* buf = nullptr;
      const size_t xb = (size_t)(g->nbc + 1) * 8;
      const size_t yb = sizeof(int) * (size_t)(g->nrows > 0 ? g->nrows : 1) + 8;
      if (cudaMalloc(&buf, xb + yb) != cudaSuccess) {
        gbo_graph_free(g);
        st = fail(GBO_ERR_NOMEM, "tuner buffers");
        break;
      }
      char* x = static_cast<char*>(buf);
      char* y = x + xb;
      cudaMemsetAsync(x, 0x55, xb, s);  // every other vertex set
      auto run = [&]() -> int {
        int d = 0;
        switch (op) {
          case GBO_TUNE_BMV: return gbo_bmv_count(g, x, y, GBO_OUT_I32, 0, stream);
          case GBO_TUNE_BFS: return gbo_bfs(g, 0, reinterpret_cast<int32_t*>(y), &d, stream);
          default: return gbo_tc_device(g, reinterpret_cast<unsigned long long*>(y), stream);
        }
      };
      st = run();
      float ms = 0.f;
      if (st == GBO_OK) {
        cudaEventRecord(e0, s);
        for (int r = 0; r < 3 && st == GBO_OK; ++r) st = run();
        cudaEventRecord(e1, s);
        const cudaError_t e = cudaEventSynchronize(e1);
        if (st == GBO_OK && e != cudaSuccess) st = fail_cuda(e, "tuner timing");
        if (st == GBO_OK) cudaEventElapsedTime(&ms, e0, e1);
      }
      c[k] = ms / 3.0;
      cudaStreamSynchronize(s);
      cudaFree(buf);
      gbo_graph_free(g);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != GBO_OK) return st;
  }
  int best = -1;
  for (int k = 0; k < 5; ++k)
    if (c[k] < INFINITY && (op != GBO_TUNE_TC || kWidths[k] >= 8) && (best < 0 || c[k] < c[best])) best = k;
  if (cost)
    for (int k = 0; k < 5; ++k) cost[k] = c[k];
  if (best < 0) return fail(GBO_ERR_OVERFLOW, "no tile width packs this matrix");
  *best_bits = kWidths[best];
  return GBO_OK;
}
