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
// is kept), and one warp per output tile sums its 32x32 popcount dot
// products in registers (lane = row r, the B tile's column words broadcast
// by shuffles).  The count pass adds each tile's non-zero entries per row
// into the row lengths (scanned into the caller's int64 row offsets); the
// fill pass gives every tile its position in each of its rows (a walk over
// the block row's tiles in column order) and writes the entries, columns
// ascending.  Block rows are processed in ranges whose pair lists fit a
// fixed budget.
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

// Block row of every A tile.
__global__ void k_tile_rows(const int* __restrict__ rowptr, int nbr, int* __restrict__ trow) {
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long I = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; I < nbr; I += nwarps)
    for (int t = rowptr[I] + (int)lane; t < rowptr[I + 1]; t += 32) trow[t] = (int)I;
}

// Pairs of A tiles [ta0, ta1) (warp per A tile, lanes over its B tiles): key
// (I, C), value (A tile, B tile); positions from the per-A-tile prefix,
// relative to the range's first pair.
__global__ void k_expand_pairs(const int* __restrict__ a_trow, const int* __restrict__ a_colind,
                               const int* __restrict__ b_rowptr, const int* __restrict__ b_colind,
                               const long long* __restrict__ pfx, long long ta0, long long ta1,
                               long long base, unsigned long long* __restrict__ keys,
                               unsigned long long* __restrict__ vals) {
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long ta = ta0 + (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5); ta < ta1; ta += nwarps) {
    const unsigned long long I = (unsigned)a_trow[ta];
    const int K = a_colind[ta];
    const int s0 = b_rowptr[K], s1 = b_rowptr[K + 1];
    const long long o = pfx[ta] - base - s0;
    for (int tb = s0 + (int)lane; tb < s1; tb += 32) {
      keys[o + tb] = (I << 32) | (unsigned)b_colind[tb];
      vals[o + tb] = ((unsigned long long)ta << 32) | (unsigned)tb;
    }
  }
}

// Output tiles of the sorted pairs: head[p] = 1 where a new key starts.
__global__ void k_group_heads(const unsigned long long* __restrict__ keys, long long np,
                              int* __restrict__ head) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np;
       p += (long long)gridDim.x * blockDim.x)
    head[p] = p == 0 || keys[p] != keys[p - 1];
}

__global__ void k_group_starts(const int* __restrict__ head, const int* __restrict__ gid, long long np,
                               int* __restrict__ gstart) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np;
       p += (long long)gridDim.x * blockDim.x)
    if (head[p]) gstart[gid[p]] = (int)p;
}

// The 32x32 product of output tile g: lane r gets row r's 32 sums.
__device__ __forceinline__ void tile_product(const unsigned* __restrict__ a_val, const unsigned* __restrict__ b_val,
                                             const unsigned long long* __restrict__ vals, int p0, int p1,
                                             unsigned lane, int (&acc)[32]) {
#pragma unroll
  for (int k = 0; k < 32; ++k) acc[k] = 0;
  for (int q = p0; q < p1; ++q) {
    const unsigned long long pv = vals[q];
    const long long ta = (long long)(pv >> 32), tb = (long long)(pv & 0xffffffffull);
    const unsigned a = a_val[ta * 32 + lane];   // row word r of A_IK
    const unsigned bw = b_val[tb * 32 + lane];  // column word c = lane of B_KC
#pragma unroll
    for (int k = 0; k < 32; ++k) acc[k] += __popc(a & __shfl_sync(0xffffffffu, bw, k));
  }
}

// Count kernel (warp per output tile): non-zero entries per row of the tile
// (cnt[g][r]) and, added up, per row of C.
__global__ void k_tile_counts(const unsigned* __restrict__ a_val, const unsigned* __restrict__ b_val,
                              const unsigned long long* __restrict__ keys,
                              const unsigned long long* __restrict__ vals, const int* __restrict__ gstart,
                              int ngroups, int nrows, int* __restrict__ cnt, int* __restrict__ rowcnt) {
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long g = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ngroups; g += nwarps) {
    const int p0 = gstart[g], p1 = gstart[g + 1];
    int acc[32];
    tile_product(a_val, b_val, vals, p0, p1, lane, acc);
    int c = 0;
#pragma unroll
    for (int k = 0; k < 32; ++k) c += acc[k] != 0;
    const long long row = (long long)(keys[p0] >> 32) * 32 + lane;
    if (row >= nrows) c = 0;
    cnt[g * 32 + lane] = c;
    if (rowcnt && c) atomicAdd(rowcnt + row, c);
  }
}

// Per block row of the range (warp, lane = row): each output tile's first
// position in its rows relative to the row's start, walking the block row's
// tiles in column order; it replaces the tile's count in place.
__global__ void k_tile_offsets(const long long* __restrict__ pfx, const int* __restrict__ a_rowptr,
                               const int* __restrict__ gid, int I0, int I1, long long base,
                               int* __restrict__ cnt) {
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long I = I0 + (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5); I < I1; I += nwarps) {
    const long long p0 = pfx[a_rowptr[I]] - base, p1 = pfx[a_rowptr[I + 1]] - base;
    if (p0 >= p1) continue;
    const int g0 = gid[p0], g1 = gid[p1];  // gid: exclusive count of heads, gid[np] = G
    int rel = 0;
    for (int g = g0; g < g1; ++g) {
      const int c = cnt[(long long)g * 32 + lane];
      cnt[(long long)g * 32 + lane] = rel;
      rel += c;
    }
  }
}

// Fill kernel (warp per output tile): the non-zero entries of row r of the
// tile at rowptr[row] + its offset, columns ascending.
__global__ void k_tile_fill(const unsigned* __restrict__ a_val, const unsigned* __restrict__ b_val,
                            const unsigned long long* __restrict__ keys,
                            const unsigned long long* __restrict__ vals, const int* __restrict__ gstart,
                            int ngroups, int nrows, const int* __restrict__ off,
                            const long long* __restrict__ rowptr, int* __restrict__ colind_out,
                            int* __restrict__ val_out) {
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long g = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ngroups; g += nwarps) {
    const int p0 = gstart[g], p1 = gstart[g + 1];
    int acc[32];
    tile_product(a_val, b_val, vals, p0, p1, lane, acc);
    const unsigned long long key = keys[p0];
    const long long row = (long long)(key >> 32) * 32 + lane;
    if (row >= nrows) continue;
    const int C = (int)(key & 0xffffffffull);
    long long pos = rowptr[row] + off[g * 32 + lane];
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      if (acc[k]) {
        colind_out[pos] = C * 32 + k;
        val_out[pos] = acc[k];
        ++pos;
      }
    }
  }
}

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
    GBO_CUDA_TRY(pool_malloc_async(&p, bytes ? bytes : 1, st));
    return GBO_OK;
  }
};

constexpr long long kPairBudget = 1ll << 25;  // tile pairs per range (keys and values: 1 GB with the sort's second buffer)

int check_pair(const gbo_graph* a, const gbo_graph* b) {
  if (!a || !b) return fail(GBO_ERR_INVALID, "NULL graph");
  if (a->b != b->b) return fail(GBO_ERR_INVALID, "A and B must have the same tile width");
  if (a->ncols != b->nrows) return fail(GBO_ERR_INVALID, "A.ncols must equal B.nrows");
  return GBO_OK;
}

// Count (fill = false: per-row entry counts into rowcnt) or fill pass of
// the sparse product.
int spgemm_pass(const gbo_graph* a, const gbo_graph* b, bool fill, int* rowcnt, const long long* rowptr,
                int* colind_out, int* val_out, cudaStream_t s) {
  if (a->b != 32 || a->layout != GBO_LAYOUT_ROW || b->layout != GBO_LAYOUT_COL)
    return fail(GBO_ERR_UNSUPPORTED, "sparse-output product: A with 32x32 ROW tiles, B with 32x32 COL tiles");
  const long long na = a->nblk;
  DevBuf cnt, pfx, tot, trow;
  GBO_TRY(cnt.alloc(sizeof(int) * (size_t)std::max(na, 1ll), s));
  GBO_TRY(pfx.alloc(sizeof(long long) * ((size_t)na + 1), s));
  GBO_TRY(tot.alloc(sizeof(long long), s));
  GBO_TRY(trow.alloc(sizeof(int) * (size_t)std::max(na, 1ll), s));
  int* d_cnt = static_cast<int*>(cnt.p);
  long long* d_pfx = static_cast<long long*>(pfx.p);
  int* d_trow = static_cast<int*>(trow.p);
  const int wgrid = 8 * num_sms();  // blocks of 8 warps, grid-stride
  if (na > 0) {
    k_pair_counts<<<(unsigned)std::min<long long>((na + 255) / 256, 4096), 256, 0, s>>>(
        a->colind, na, b->rowptr, d_cnt);
    k_tile_rows<<<wgrid, 256, 0, s>>>(a->rowptr, a->nbr, d_trow);
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
  DevBuf kbuf[2], vbuf[2], temp, head, gid, gstart, tcnt, ng;
  size_t temp_bytes = 0;
  long long tcap = 0;  // output tiles the per-tile counts can hold
  GBO_TRY(ng.alloc(sizeof(long long), s));
  for (int I0 = 0; I0 < a->nbr;) {
    int I1 = I0 + 1;
    while (I1 < a->nbr && hp[arp[I1 + 1]] - hp[arp[I0]] <= kPairBudget) ++I1;
    const long long base = hp[arp[I0]], np = hp[arp[I1]] - base;
    if (np > 2147483647LL) return fail(GBO_ERR_OVERFLOW, "one block row has more than 2^31-1 tile pairs");
    if (np > 0) {
      if (np > cap) {
        for (int k = 0; k < 2; ++k) {
          GBO_TRY(kbuf[k].alloc(sizeof(unsigned long long) * (size_t)np, s));
          GBO_TRY(vbuf[k].alloc(sizeof(unsigned long long) * (size_t)np, s));
        }
        GBO_TRY(head.alloc(sizeof(int) * (size_t)np, s));
        GBO_TRY(gid.alloc(sizeof(int) * ((size_t)np + 1), s));
        GBO_TRY(gstart.alloc(sizeof(int) * ((size_t)np + 1), s));
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
      int* d_head = static_cast<int*>(head.p);
      int* d_gid = static_cast<int*>(gid.p);
      int* d_gstart = static_cast<int*>(gstart.p);
      k_expand_pairs<<<wgrid, 256, 0, s>>>(d_trow, a->colind, b->rowptr, b->colind, d_pfx, arp[I0], arp[I1],
                                           base, k0, v0);
      GBO_CUDA_TRY(cudaGetLastError());
      size_t tb = temp_bytes;
      GBO_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.p, tb, k0, k1, v0, v1, (int)np, 0, 64, s));
      // output tiles: heads, their ids (exclusive scan) and first pairs
      const unsigned eg = (unsigned)std::min<long long>((np + 255) / 256, 8192);
      k_group_heads<<<eg, 256, 0, s>>>(k1, np, d_head);
      GBO_TRY(exclusive_scan_i32(d_head, d_gid, np, static_cast<long long*>(ng.p), s));
      k_group_starts<<<eg, 256, 0, s>>>(d_head, d_gid, np, d_gstart);
      GBO_CUDA_TRY(cudaGetLastError());
      // d_gid[np] is the number of output tiles; gstart[G] = np
      int G = 0;
      GBO_CUDA_TRY(cudaMemcpyAsync(&G, d_gid + np, sizeof(int), cudaMemcpyDeviceToHost, s));
      GBO_CUDA_TRY(cudaStreamSynchronize(s));
      const int npi = (int)np;
      GBO_CUDA_TRY(cudaMemcpyAsync(d_gstart + G, &npi, sizeof(int), cudaMemcpyHostToDevice, s));
      if (G > tcap) {
        GBO_TRY(tcnt.alloc(sizeof(int) * 32 * (size_t)G, s));
        tcap = G;
      }
      int* d_tcnt = static_cast<int*>(tcnt.p);
      const auto* av = static_cast<const unsigned*>(a->val);
      const auto* bv = static_cast<const unsigned*>(b->val);
      k_tile_counts<<<wgrid, 256, 0, s>>>(av, bv, k1, v1, d_gstart, G, a->nrows, d_tcnt, fill ? nullptr : rowcnt);
      if (fill) {
        k_tile_offsets<<<wgrid, 256, 0, s>>>(d_pfx, a->rowptr, d_gid, I0, I1, base, d_tcnt);
        k_tile_fill<<<wgrid, 256, 0, s>>>(av, bv, k1, v1, d_gstart, G, a->nrows, d_tcnt, rowptr, colind_out,
                                          val_out);
      }
      GBO_CUDA_TRY(cudaGetLastError());
      GBO_CUDA_TRY(cudaStreamSynchronize(s));  // npi lives on this frame
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
