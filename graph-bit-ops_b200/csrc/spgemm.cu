// Unmasked binary matrix products on B2SR: the total of A B
// (bmm{4,8,16,32,64}_sparse, bsrbmm/bsrbmm.cu:244-555) and A B with sparse
// output (bmm32_sparse_symbolic / bmm32_sparse_numeric,
// bsrbmm/bsrbmm.cu:1273-1373).
//
// Total.  The reference forms every tile product A_IK B_KC and adds all
// its entries.  The sum of the entries of A B is sum_m colcount_A(m) *
// rowcount_B(m), so here one pass over each operand's tile words gives the
// two line counts and a dot product gives the total: the same integer at
// the cost of reading the operands once.
//
// Sparse output (32x32 tiles, A with row words, B with column words as in
// the reference: entry (r, c) of A_IK B_KC is popc(A_IK[r] & B_KC[c])).
// The reference's numeric kernel tries every block column for every block
// row (a binary search per (block column, A tile)); here the tile pairs are
// enumerated instead: every A tile (I, K) meets every B tile (K, C), the
// pairs are sorted by output tile (I, C) (stable, so the K order of a tile
// is kept), and one warp per block row walks its pairs in output-tile order,
// summing 32x32 popcount dot products in registers (lane = row r, the B
// tile's column words broadcast by shuffles) and emitting the non-zero
// entries of each output tile in column order.  A count pass gives the row
// lengths (scanned into the caller's int64 row offsets); a fill pass writes
// column indices and counts.  Block rows are processed in ranges whose pair
// lists fit a fixed budget.
#include <algorithm>
#include <vector>

#include <cub/cub.cuh>

#include "bmv.cuh"

namespace gbo {
namespace {

// ------------------------------------------------------------ line counts
// Row and column counts of a B2SR matrix: word q of tile t is tile row q
// (ROW layout) or tile column q (COL layout); its popcount adds to that line,
// and its set bits add one each to the crossing lines.
template <int B>
__global__ void k_line_counts(GView v, int layout, unsigned long long* __restrict__ rows,
                              unsigned long long* __restrict__ cols) {
  using WT = typename Word<B>::T;
  const WT* __restrict__ val = reinterpret_cast<const WT*>(v.val);
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long item = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; item < v.nitems;
       item += nwarps) {
    const gbo_item it = v.items[item];
    for (long long q = (long long)it.t0 * B + lane; q < (long long)it.t1 * B; q += 32) {
      const long long t = q / B;
      const int w = (int)(q % B);
      unsigned long long word = (unsigned long long)val[q];
      if (B == 4) word &= 0xfull;
      if (!word) continue;
      const long long R = (long long)it.row * B, C = (long long)v.colind[t] * B;
      const long long line = (layout == GBO_LAYOUT_ROW ? R : C) + w;     // the word's own line
      const long long cross = layout == GBO_LAYOUT_ROW ? C : R;           // lines its bits cross
      unsigned long long* own = layout == GBO_LAYOUT_ROW ? rows : cols;
      unsigned long long* other = layout == GBO_LAYOUT_ROW ? cols : rows;
      if (own) atomicAdd(own + line, (unsigned long long)__popcll(word));
      if (other) {
        while (word) {
          const int hi = 63 - __clzll((long long)word);  // bit position from the low end
          word &= ~(1ull << hi);
          atomicAdd(other + cross + (B - 1 - hi), 1ull);
        }
      }
    }
  }
}

__global__ void k_dot_counts(const unsigned long long* __restrict__ a,
                             const unsigned long long* __restrict__ b, long long n,
                             unsigned long long* __restrict__ out) {
  unsigned long long s = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    s += a[i] * b[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

int launch_line_counts(const gbo_graph* g, unsigned long long* rows, unsigned long long* cols,
                       cudaStream_t s) {
  if (g->nitems <= 0) return GBO_OK;
  GView v = view_of(g);
  const int grid = (int)std::min<long long>(((long long)g->nitems + 7) / 8, 8LL * num_sms());
  switch (g->b) {
    case 4: k_line_counts<4><<<grid, 256, 0, s>>>(v, g->layout, rows, cols); break;
    case 8: k_line_counts<8><<<grid, 256, 0, s>>>(v, g->layout, rows, cols); break;
    case 16: k_line_counts<16><<<grid, 256, 0, s>>>(v, g->layout, rows, cols); break;
    case 32: k_line_counts<32><<<grid, 256, 0, s>>>(v, g->layout, rows, cols); break;
    default: k_line_counts<64><<<grid, 256, 0, s>>>(v, g->layout, rows, cols); break;
  }
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

// --------------------------------------------------------- sparse output
// Tile pairs of each A tile: |B block row colA[t]|.
__global__ void k_pair_counts(const int* __restrict__ a_colind, long long nblk_a,
                              const int* __restrict__ b_rowptr, int* __restrict__ cnt) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nblk_a;
       t += (long long)gridDim.x * blockDim.x) {
    const int K = a_colind[t];
    cnt[t] = b_rowptr[K + 1] - b_rowptr[K];
  }
}

// Pairs of block rows [I0, I1): key (I, C), value (A tile, B tile); pair
// positions from the per-A-tile prefix (relative to the range's first pair).
__global__ void k_expand_pairs(const int* __restrict__ a_rowptr, const int* __restrict__ a_colind,
                               const int* __restrict__ b_rowptr, const int* __restrict__ b_colind,
                               const long long* __restrict__ pfx, int I0, int I1, long long base,
                               unsigned long long* __restrict__ keys,
                               unsigned long long* __restrict__ vals) {
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long I = I0 + (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5); I < I1; I += nwarps) {
    for (int ta = a_rowptr[I]; ta < a_rowptr[I + 1]; ++ta) {
      const int K = a_colind[ta];
      const int s0 = b_rowptr[K], s1 = b_rowptr[K + 1];
      const long long o = pfx[ta] - base - s0;
      for (int tb = s0 + (int)lane; tb < s1; tb += 32) {
        keys[o + tb] = ((unsigned long long)I << 32) | (unsigned)b_colind[tb];
        vals[o + tb] = ((unsigned long long)ta << 32) | (unsigned)tb;
      }
    }
  }
}

// One warp per block row of the range: walk its sorted pairs, one output
// tile (equal keys) at a time; lane r sums row r of the tile's product.
// FILL = false: per-row entry counts; FILL = true: entries at the row
// offsets.
template <bool FILL>
__global__ void k_tile_products(const unsigned* __restrict__ a_val, const unsigned* __restrict__ b_val,
                                const long long* __restrict__ pfx, const int* __restrict__ a_rowptr,
                                int I0, int I1, long long base, int nrows,
                                const unsigned long long* __restrict__ keys,
                                const unsigned long long* __restrict__ vals,
                                int* __restrict__ rowcnt, const long long* __restrict__ rowptr,
                                int* __restrict__ colind_out, int* __restrict__ val_out) {
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long I = I0 + (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5); I < I1; I += nwarps) {
    const long long p0 = pfx[a_rowptr[I]] - base, p1 = pfx[a_rowptr[I + 1]] - base;
    const long long row = I * 32 + lane;
    int cnt_row = 0;
    long long pos = FILL && row < nrows ? rowptr[row] : 0;
    long long p = p0;
    while (p < p1) {
      const unsigned C = (unsigned)(keys[p] & 0xffffffffull);
      int acc[32];
#pragma unroll
      for (int k = 0; k < 32; ++k) acc[k] = 0;
      long long q = p;
      for (; q < p1 && (unsigned)(keys[q] & 0xffffffffull) == C; ++q) {
        const unsigned long long pv = vals[q];
        const long long ta = (long long)(pv >> 32), tb = (long long)(pv & 0xffffffffull);
        const unsigned a = a_val[ta * 32 + lane];   // row word r of A_IK
        const unsigned bw = b_val[tb * 32 + lane];  // column word c = lane of B_KC
#pragma unroll
        for (int k = 0; k < 32; ++k) acc[k] += __popc(a & __shfl_sync(0xffffffffu, bw, k));
      }
      if (row < nrows) {
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          if (acc[k]) {
            if (FILL) {
              colind_out[pos] = (int)(C * 32 + k);
              val_out[pos] = acc[k];
              ++pos;
            } else {
              ++cnt_row;
            }
          }
        }
      }
      p = q;
    }
    if (!FILL && row < nrows) rowcnt[row] = cnt_row;
  }
}

// Stream-ordered device buffer freed on scope exit (alloc replaces it).
struct DevBuf {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
  }
  int alloc(size_t bytes, cudaStream_t st) {
    release();
    s = st;
    GBO_CUDA_TRY(cudaMallocAsync(&p, bytes ? bytes : 1, st));
    return GBO_OK;
  }
};

constexpr long long kPairBudget = 1ll << 25;  // tile pairs per range (512 MB of keys and values)

int check_pair(const gbo_graph* a, const gbo_graph* b) {
  if (!a || !b) return fail(GBO_ERR_INVALID, "NULL graph");
  if (a->b != b->b) return fail(GBO_ERR_INVALID, "A and B must have the same tile width");
  if (a->ncols != b->nrows) return fail(GBO_ERR_INVALID, "A.ncols must equal B.nrows");
  return GBO_OK;
}

// Count (FILL = false) or fill pass of the sparse product.
int spgemm_pass(const gbo_graph* a, const gbo_graph* b, bool fill, int* rowcnt, const long long* rowptr,
                int* colind_out, int* val_out, cudaStream_t s) {
  if (a->b != 32 || a->layout != GBO_LAYOUT_ROW || b->layout != GBO_LAYOUT_COL)
    return fail(GBO_ERR_UNSUPPORTED, "sparse-output product: A with 32x32 ROW tiles, B with 32x32 COL tiles");
  const long long na = a->nblk;
  DevBuf cnt, pfx, tot;
  GBO_TRY(cnt.alloc(sizeof(int) * (size_t)std::max(na, 1ll), s));
  GBO_TRY(pfx.alloc(sizeof(long long) * ((size_t)na + 1), s));
  GBO_TRY(tot.alloc(sizeof(long long), s));
  int* d_cnt = static_cast<int*>(cnt.p);
  long long* d_pfx = static_cast<long long*>(pfx.p);
  if (na > 0) {
    k_pair_counts<<<(unsigned)std::min<long long>((na + 255) / 256, 4096), 256, 0, s>>>(
        a->colind, na, b->rowptr, d_cnt);
    GBO_CUDA_TRY(cudaGetLastError());
  }
  GBO_TRY(exclusive_scan_i32_to_i64(d_cnt, d_pfx, na, static_cast<long long*>(tot.p), s));
  // block-row ranges whose pairs fit the budget (host copies of the offsets)
  std::vector<int> arp((size_t)a->nbr + 1);
  std::vector<long long> hp((size_t)na + 1);
  GBO_CUDA_TRY(cudaMemcpyAsync(arp.data(), a->rowptr, sizeof(int) * arp.size(), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaMemcpyAsync(hp.data(), d_pfx, sizeof(long long) * hp.size(), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  if (!fill && a->nrows > 0) GBO_CUDA_TRY(cudaMemsetAsync(rowcnt, 0, sizeof(int) * (size_t)a->nrows, s));
  long long cap = 0;
  DevBuf kbuf[2], vbuf[2], temp;
  size_t temp_bytes = 0;
  for (int I0 = 0; I0 < a->nbr;) {
    int I1 = I0 + 1;
    while (I1 < a->nbr && hp[arp[I1 + 1]] - hp[arp[I0]] <= kPairBudget) ++I1;
    const long long base = hp[arp[I0]], np = hp[arp[I1]] - base;
    if (np > 0) {
      if (np > cap) {
        for (int k = 0; k < 2; ++k) {
          GBO_TRY(kbuf[k].alloc(sizeof(unsigned long long) * (size_t)np, s));
          GBO_TRY(vbuf[k].alloc(sizeof(unsigned long long) * (size_t)np, s));
        }
        cap = np;
        size_t need = 0;
        GBO_CUDA_TRY(cub::DeviceRadixSort::SortPairs(
            nullptr, need, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
            (unsigned long long*)nullptr, (unsigned long long*)nullptr, (int)np, 0, 64, s));
        if (need > temp_bytes) {
          GBO_TRY(temp.alloc(need, s));
          temp_bytes = need;
        }
      }
      auto* k0 = static_cast<unsigned long long*>(kbuf[0].p);
      auto* v0 = static_cast<unsigned long long*>(vbuf[0].p);
      auto* k1 = static_cast<unsigned long long*>(kbuf[1].p);
      auto* v1 = static_cast<unsigned long long*>(vbuf[1].p);
      const int nrow = I1 - I0;
      const int grid = (int)std::min<long long>(((long long)nrow + 7) / 8, 8LL * num_sms());
      k_expand_pairs<<<grid, 256, 0, s>>>(a->rowptr, a->colind, b->rowptr, b->colind, d_pfx, I0, I1, base,
                                          k0, v0);
      GBO_CUDA_TRY(cudaGetLastError());
      size_t tb = temp_bytes;
      GBO_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.p, tb, k0, k1, v0, v1, (int)np, 0, 64, s));
      if (fill)
        k_tile_products<true><<<grid, 256, 0, s>>>(static_cast<const unsigned*>(a->val),
                                                   static_cast<const unsigned*>(b->val), d_pfx, a->rowptr,
                                                   I0, I1, base, a->nrows, k1, v1, nullptr, rowptr,
                                                   colind_out, val_out);
      else
        k_tile_products<false><<<grid, 256, 0, s>>>(static_cast<const unsigned*>(a->val),
                                                    static_cast<const unsigned*>(b->val), d_pfx, a->rowptr,
                                                    I0, I1, base, a->nrows, k1, v1, rowcnt, nullptr, nullptr,
                                                    nullptr);
      GBO_CUDA_TRY(cudaGetLastError());
    }
    I0 = I1;
  }
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  return GBO_OK;
}

}  // namespace
}  // namespace gbo

using namespace gbo;

extern "C" int gbo_bmm_sum(const gbo_graph* a, const gbo_graph* b, uint64_t* h_sum, gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_pair(a, b));
  if (!h_sum) return fail(GBO_ERR_INVALID, "h_sum is NULL");
  cudaStream_t s = as_stream(stream);
  const long long n = a->ncols;  // the shared dimension
  DevBuf buf;
  GBO_TRY(buf.alloc(sizeof(unsigned long long) * (2 * (size_t)n + 1), s));
  auto* colA = static_cast<unsigned long long*>(buf.p);
  auto* rowB = colA + n;
  auto* out = rowB + n;
  GBO_CUDA_TRY(cudaMemsetAsync(buf.p, 0, sizeof(unsigned long long) * (2 * (size_t)n + 1), s));
  GBO_TRY(launch_line_counts(a, nullptr, colA, s));
  GBO_TRY(launch_line_counts(b, rowB, nullptr, s));
  if (n > 0) {
    k_dot_counts<<<(unsigned)std::min<long long>((n + 255) / 256, 4096), 256, 0, s>>>(colA, rowB, n, out);
    GBO_CUDA_TRY(cudaGetLastError());
  }
  unsigned long long h = 0;
  GBO_CUDA_TRY(cudaMemcpyAsync(&h, out, sizeof(h), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  *h_sum = h;
  return GBO_OK;
}

extern "C" int gbo_spgemm_nnz(const gbo_graph* a, const gbo_graph* b, int64_t* d_rowptr, int64_t* h_nnz,
                              gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_pair(a, b));
  if (!d_rowptr) return fail(GBO_ERR_INVALID, "d_rowptr is NULL");
  cudaStream_t s = as_stream(stream);
  DevBuf cnt, tot;
  GBO_TRY(cnt.alloc(sizeof(int) * (size_t)std::max(a->nrows, 1), s));
  GBO_TRY(tot.alloc(sizeof(long long), s));
  GBO_TRY(spgemm_pass(a, b, false, static_cast<int*>(cnt.p), nullptr, nullptr, nullptr, s));
  GBO_TRY(exclusive_scan_i32_to_i64(static_cast<int*>(cnt.p), reinterpret_cast<long long*>(d_rowptr),
                                    a->nrows, static_cast<long long*>(tot.p), s));
  long long nnz = 0;
  GBO_CUDA_TRY(cudaMemcpyAsync(&nnz, tot.p, sizeof(nnz), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  if (h_nnz) *h_nnz = nnz;
  return GBO_OK;
}

extern "C" int gbo_spgemm_fill(const gbo_graph* a, const gbo_graph* b, const int64_t* d_rowptr,
                               int32_t* d_colind, int32_t* d_val, gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_pair(a, b));
  if (!d_rowptr || !d_colind || !d_val) return fail(GBO_ERR_INVALID, "NULL output");
  return spgemm_pass(a, b, true, nullptr, reinterpret_cast<const long long*>(d_rowptr), d_colind, d_val,
                     as_stream(stream));
}
