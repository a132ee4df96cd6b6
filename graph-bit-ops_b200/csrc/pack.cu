// B2SR packing on the device (replaces the host-serial csr2bsr_batch_*,
// algorithm/csr2bsr_batch_bsrbmv.cu:9-946, and bsrbmm/csr2bsr_batch.cu).
//
// The reference walks block rows on the host, runs cuSPARSE csr2bsr into a
// dense float b x b buffer per slab and packs it with ToBit*Col.  Here one
// warp lane owns one CSR row of a slab of b rows (b <= 32: 32/b slabs per
// warp; b = 64: each lane owns rows r and r+32).  Because CSR rows are
// sorted, the slab's tiles come out in ascending block-column order by a
// b-way merge: every step takes the smallest head block column m over the
// slab's rows (a segmented shuffle min), each lane ORs the bits of all its
// entries in block column m into its tile row word, and the group emits one
// tile.  A count pass sizes each block row; a scan gives bsrRowPtr; a fill
// pass writes bsrColInd and the tile words (one coalesced store of b words).
#include <vector>
#include <algorithm>
#include "graph.cuh"

namespace gbo {

namespace {

constexpr int kPackTPB = 256;

template <int B>
struct SlabMap {
  // lanes per slab and slabs per warp
  static constexpr int W = B >= 32 ? 32 : B;
  static constexpr int G = 32 / W;
  static constexpr int RPL = B > 32 ? 2 : 1;  // rows per lane
};

__device__ __forceinline__ int seg_min(int v, int width) {
  for (int o = width >> 1; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Per-lane cursor over one CSR row.
struct RowCursor {
  long long pos, end;
  int prev;
};

__device__ __forceinline__ void init_cursor(RowCursor& c, const int* __restrict__ rowptr, int row,
                                            int nrows, long long nnz, unsigned* derr) {
  c.pos = 0;
  c.end = 0;
  c.prev = -1;
  if (row < nrows) {
    long long a = rowptr[row], e = rowptr[row + 1];
    if (a < 0 || e < a || e > nnz) {
      atomicOr(derr, DERR_ROWPTR);
    } else {
      c.pos = a;
      c.end = e;
    }
  }
}

template <int B>
__device__ __forceinline__ int head_of(const RowCursor& c, const int* __restrict__ colind) {
  return c.pos < c.end ? colind[c.pos] / B : kINF;
}

// Consume all entries of block column m from the cursor; OR their bits.
template <int B, typename WT>
__device__ __forceinline__ void consume(RowCursor& c, const int* __restrict__ colind, int m,
                                        int ncols, WT& word, unsigned* derr, bool build) {
  while (c.pos < c.end) {
    int col = colind[c.pos];
    if (col / B != m) break;
    if (col < c.prev) atomicOr(derr, DERR_UNSORTED);
    if (col < 0 || col >= ncols) atomicOr(derr, DERR_COL_BOUNDS);
    c.prev = col;
    if (build) word |= (WT)((WT)1 << (B - 1 - ((unsigned)col % B)));
    ++c.pos;
  }
}

// After a lane's row ends, any remaining (unsorted) entries are still
// consumed by the merge; a head < previous column marks the row unsorted.
template <int B>
__device__ __forceinline__ void check_head(const RowCursor& c, const int* __restrict__ colind,
                                           unsigned* derr) {
  if (c.pos < c.end && c.prev >= 0 && colind[c.pos] < c.prev) atomicOr(derr, DERR_UNSORTED);
}

// COUNT (build=false) and FILL (build=true) share one body.
template <int B, bool BUILD>
__global__ void __launch_bounds__(kPackTPB) k_pack(const int* __restrict__ rowptr,
                                                   const int* __restrict__ colind, int nrows,
                                                   int ncols, long long nnz, int nbr,
                                                   int* __restrict__ counts,
                                                   const int* __restrict__ bsr_rowptr,
                                                   int* __restrict__ bsr_colind,
                                                   typename Word<B>::T* __restrict__ bsr_val,
                                                   int layout, unsigned* derr) {
  using WT = typename Word<B>::T;
  using M = SlabMap<B>;
  const unsigned lane = threadIdx.x & 31;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int g = lane / M::W;          // slab within warp
  const int r = lane % M::W;          // row within slab (first row for B=64)
  const long long slab = warp * M::G + g;
  if (warp * M::G >= nbr) return;     // whole warp idle (uniform)
  const bool slab_ok = slab < nbr;

  RowCursor c0, c1;
  const long long row0 = slab * B + r;
  init_cursor(c0, rowptr, slab_ok && row0 < nrows ? (int)row0 : nrows, nrows, nnz, derr);
  if (M::RPL == 2) {
    const long long row1 = slab * B + 32 + r;
    init_cursor(c1, rowptr, slab_ok && row1 < nrows ? (int)row1 : nrows, nrows, nnz, derr);
  }

  long long out = 0;
  if (BUILD && slab_ok) out = bsr_rowptr[slab];
  int ntile = 0;

  while (true) {
    int h = head_of<B>(c0, colind);
    if (M::RPL == 2) h = min(h, head_of<B>(c1, colind));
    const int m = seg_min(h, M::W);
    if (!__any_sync(0xffffffffu, m != kINF)) break;
    WT w0 = 0, w1 = 0;
    if (m != kINF) {
      consume<B, WT>(c0, colind, m, ncols, w0, derr, BUILD);
      check_head<B>(c0, colind, derr);
      if (M::RPL == 2) {
        consume<B, WT>(c1, colind, m, ncols, w1, derr, BUILD);
        check_head<B>(c1, colind, derr);
      }
    }
    if (BUILD) {
      const long long tile = out + ntile;
      if (layout == GBO_LAYOUT_ROW) {
        if (m != kINF) {
          if (r == 0) bsr_colind[tile] = m;
          bsr_val[tile * B + r] = w0;
          if (M::RPL == 2) bsr_val[tile * B + 32 + r] = w1;
        }
      } else {
        // transpose the b x b bit tile with ballots: column word c has row r
        // at bit (b-1-r).
        if (M::RPL == 1) {
          WT mine = 0;
#pragma unroll 4
          for (int cc = 0; cc < B; ++cc) {
            unsigned bal = __ballot_sync(0xffffffffu, (w0 >> (B - 1 - cc)) & 1);
            unsigned seg = (bal >> (g * M::W)) & seg_mask<B>();
            unsigned colw = __brev(seg) >> (32 - (B < 32 ? B : 32));
            if (r == cc) mine = (WT)colw;
          }
          if (m != kINF) {
            if (r == 0) bsr_colind[tile] = m;
            bsr_val[tile * B + r] = mine;
          }
        } else {
          unsigned long long lo_w = 0, hi_w = 0;
#pragma unroll 4
          for (int cc = 0; cc < 64; ++cc) {
            unsigned lo = __ballot_sync(0xffffffffu, (unsigned)((w0 >> (63 - cc)) & 1ull));
            unsigned hi = __ballot_sync(0xffffffffu, (unsigned)((w1 >> (63 - cc)) & 1ull));
            unsigned long long colw = __brevll(((unsigned long long)hi << 32) | lo);
            if (cc == (int)r) lo_w = colw;
            if (cc == (int)r + 32) hi_w = colw;
          }
          if (m != kINF) {
            if (r == 0) bsr_colind[tile] = m;
            bsr_val[tile * B + r] = (WT)lo_w;
            bsr_val[tile * B + 32 + r] = (WT)hi_w;
          }
        }
      }
    }
    if (m != kINF) ++ntile;
  }
  if (!BUILD && slab_ok && r == 0) counts[slab] = ntile;
}

// ---------------------------------------------------------------- scan
constexpr int kScanTPB = 1024;

__global__ void k_scan_block_sums(const int* __restrict__ in, long long n,
                                  long long* __restrict__ sums) {
  __shared__ long long sh[32];
  long long i = (long long)blockIdx.x * kScanTPB + threadIdx.x;
  long long v = i < n ? in[i] : 0;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    long long s = sh[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) sums[blockIdx.x] = s;
  }
}

// Exclusive scan of up to kScanTPB*kScanTPB block sums by one block (loop).
__global__ void k_scan_sums(long long* __restrict__ sums, long long nb, long long* total) {
  __shared__ long long sh[32];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (long long base = 0; base < nb; base += kScanTPB) {
    long long i = base + threadIdx.x;
    long long v = i < nb ? sums[i] : 0;
    // inclusive warp scan
    long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, x, o);
      if ((threadIdx.x & 31) >= (unsigned)o) x += y;
    }
    if ((threadIdx.x & 31) == 31) sh[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
      long long s = sh[threadIdx.x];
      for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, s, o);
        if (threadIdx.x >= (unsigned)o) s += y;
      }
      sh[threadIdx.x] = s;
    }
    __syncthreads();
    long long warp_prefix = (threadIdx.x >> 5) ? sh[(threadIdx.x >> 5) - 1] : 0;
    long long incl = x + warp_prefix + carry;
    if (i < nb) sums[i] = incl - v;
    __syncthreads();
    if (threadIdx.x == kScanTPB - 1) carry = incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

template <typename OutT>
__global__ void k_scan_apply(const int* __restrict__ in, long long n,
                             const long long* __restrict__ sums, OutT* __restrict__ out,
                             const long long* __restrict__ total) {
  __shared__ long long sh[32];
  long long i = (long long)blockIdx.x * kScanTPB + threadIdx.x;
  long long v = i < n ? in[i] : 0;
  long long x = v;
  for (int o = 1; o < 32; o <<= 1) {
    long long y = __shfl_up_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) >= (unsigned)o) x += y;
  }
  if ((threadIdx.x & 31) == 31) sh[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x < 32) {
    long long s = sh[threadIdx.x];
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, s, o);
      if (threadIdx.x >= (unsigned)o) s += y;
    }
    sh[threadIdx.x] = s;
  }
  __syncthreads();
  long long warp_prefix = (threadIdx.x >> 5) ? sh[(threadIdx.x >> 5) - 1] : 0;
  long long excl = x - v + warp_prefix + sums[blockIdx.x];
  if (sizeof(OutT) == 8) {
    if (i < n) out[i] = (OutT)excl;
    if (i == 0) out[n] = (OutT)*total;
  } else {
    if (i < n) out[i] = (OutT)(excl > 2147483647LL ? 2147483647LL : excl);
    if (i == 0) out[n] = (OutT)(*total > 2147483647LL ? 2147483647LL : *total);
  }
}

// ------------------------------------------------------- vector packing
template <int B>
__global__ void k_pack_vec(const float* __restrict__ xf, const int32_t* __restrict__ xi, int n,
                           typename Word<B>::T* __restrict__ bits, long long nwords) {
  using WT = typename Word<B>::T;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned lane = threadIdx.x & 31;
  bool v = false;
  if (i < n) v = xf ? (xf[i] > 0.f) : (xi[i] > 0);
  unsigned bal = __brev(__ballot_sync(0xffffffffu, v));  // element (base+k) at bit 31-k
  const long long base = i - lane;                        // first element of this warp
  if (B == 64) {
    // two warps make one 64-bit word: even warp -> high half, odd warp -> low half
    const long long word = base / 64;
    if (lane == 0 && word < nwords) {
      unsigned long long* wp = reinterpret_cast<unsigned long long*>(bits) + word;
      unsigned long long part = ((base / 32) & 1) ? (unsigned long long)bal
                                                  : ((unsigned long long)bal << 32);
      atomicOr(wp, part);
    }
  } else {
    constexpr int S = 32 / B;  // segments per warp chunk
    if ((int)lane < S) {
      const long long word = base / B + lane;
      if (word < nwords) {
        unsigned seg = (bal >> (32 - B * (lane + 1))) & seg_mask<B>();
        bits[word] = (WT)seg;
      }
    }
  }
}

template <int B>
__global__ void k_unpack_vec(const typename Word<B>::T* __restrict__ bits, int n,
                             int32_t* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long w = (unsigned long long)bits[i / B];
  out[i] = (int32_t)((w >> (B - 1 - (i % B))) & 1ull);
}

// ------------------------------------------------------------ out-degree
__global__ void k_col_hist(const int* __restrict__ colind, long long nnz, int ncols,
                           int* __restrict__ deg) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
       i += (long long)gridDim.x * blockDim.x) {
    int c = colind[i];
    if (c >= 0 && c < ncols) atomicAdd(deg + c, 1);
  }
}
__global__ void k_row_len(const int* __restrict__ rowptr, int nrows, int* __restrict__ deg) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nrows) deg[i] = rowptr[i + 1] - rowptr[i];
}
__global__ void k_inv(const int* __restrict__ deg, int n, float* __restrict__ inv) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) inv[i] = deg[i] > 0 ? 1.0f / (float)deg[i] : 0.0f;
}

// ------------------------------------------------------------- schedule
__global__ void k_sched_counts(const int* __restrict__ rowptr, int nbr, int chunk,
                               int* __restrict__ nchunk, int* __restrict__ nslot,
                               int* __restrict__ issplit) {
  long long R = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (R >= nbr) return;
  int len = rowptr[R + 1] - rowptr[R];
  int k = len <= chunk ? 1 : (len + chunk - 1) / chunk;
  nchunk[R] = k;
  nslot[R] = k > 1 ? k : 0;
  issplit[R] = k > 1 ? 1 : 0;
}

__global__ void k_sched_fill(const int* __restrict__ rowptr, int nbr, int chunk,
                             const int* __restrict__ item_off, const int* __restrict__ slot_off,
                             const int* __restrict__ split_off, gbo_item* __restrict__ items,
                             gbo_split* __restrict__ splits) {
  long long R = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (R >= nbr) return;
  int t0 = rowptr[R], t1 = rowptr[R + 1];
  int len = t1 - t0;
  int k = len <= chunk ? 1 : (len + chunk - 1) / chunk;
  int base = item_off[R];
  if (k == 1) {
    items[base] = gbo_item{(int)R, t0, t1, -1};
  } else {
    int s0 = slot_off[R];
    for (int q = 0; q < k; ++q) {
      int a = t0 + q * chunk;
      int e = min(t1, a + chunk);
      items[base + q] = gbo_item{(int)R, a, e, s0 + q};
    }
    splits[split_off[R]] = gbo_split{(int)R, s0, k, 0};
  }
}

template <int B>
int launch_pack(bool build, const int* rowptr, const int* colind, int nrows, int ncols,
                long long nnz, int nbr, int* counts, const int* bsr_rowptr, int* bsr_colind,
                void* bsr_val, int layout, unsigned* derr, cudaStream_t s) {
  using M = SlabMap<B>;
  long long warps = (nbr + M::G - 1) / M::G;
  unsigned grid = blocks_for_warps(warps, kPackTPB / 32);
  if (build)
    k_pack<B, true><<<grid, kPackTPB, 0, s>>>(rowptr, colind, nrows, ncols, nnz, nbr, counts,
                                              bsr_rowptr, bsr_colind,
                                              reinterpret_cast<typename Word<B>::T*>(bsr_val),
                                              layout, derr);
  else
    k_pack<B, false><<<grid, kPackTPB, 0, s>>>(rowptr, colind, nrows, ncols, nnz, nbr, counts,
                                               bsr_rowptr, bsr_colind,
                                               reinterpret_cast<typename Word<B>::T*>(bsr_val),
                                               layout, derr);
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

int dispatch_pack(int b, bool build, const int* rowptr, const int* colind, int nrows, int ncols,
                  long long nnz, int nbr, int* counts, const int* bsr_rowptr, int* bsr_colind,
                  void* bsr_val, int layout, unsigned* derr, cudaStream_t s) {
  switch (b) {
    case 4: return launch_pack<4>(build, rowptr, colind, nrows, ncols, nnz, nbr, counts, bsr_rowptr, bsr_colind, bsr_val, layout, derr, s);
    case 8: return launch_pack<8>(build, rowptr, colind, nrows, ncols, nnz, nbr, counts, bsr_rowptr, bsr_colind, bsr_val, layout, derr, s);
    case 16: return launch_pack<16>(build, rowptr, colind, nrows, ncols, nnz, nbr, counts, bsr_rowptr, bsr_colind, bsr_val, layout, derr, s);
    case 32: return launch_pack<32>(build, rowptr, colind, nrows, ncols, nnz, nbr, counts, bsr_rowptr, bsr_colind, bsr_val, layout, derr, s);
    case 64: return launch_pack<64>(build, rowptr, colind, nrows, ncols, nnz, nbr, counts, bsr_rowptr, bsr_colind, bsr_val, layout, derr, s);
  }
  return fail(GBO_ERR_INVALID, "tile_bits must be 4, 8, 16, 32 or 64");
}

int derr_to_status(unsigned e) {
  if (e & DERR_ROWPTR) return fail(GBO_ERR_BOUNDS, "CSR row pointers are not monotone within [0, nnz]");
  if (e & DERR_COL_BOUNDS) return fail(GBO_ERR_BOUNDS, "CSR column index outside [0, ncols)");
  if (e & DERR_UNSORTED) return fail(GBO_ERR_UNSORTED, "CSR column indices are not ascending inside a row");
  return GBO_OK;
}

// Small device scratch for the scan + error word, stream-ordered.
struct ScanScratch {
  long long* sums = nullptr;
  long long* total = nullptr;
  unsigned* derr = nullptr;
};

}  // namespace

namespace {
template <typename OutT>
int exclusive_scan(const int* d_in, OutT* d_out, long long n, long long* d_total, cudaStream_t s) {
  long long nb = (n + kScanTPB - 1) / kScanTPB;
  if (nb < 1) nb = 1;
  long long* sums = nullptr;
  GBO_CUDA_TRY(pool_malloc_async(&sums, sizeof(long long) * nb, s));
  k_scan_block_sums<<<(unsigned)nb, kScanTPB, 0, s>>>(d_in, n, sums);
  k_scan_sums<<<1, kScanTPB, 0, s>>>(sums, nb, d_total);
  k_scan_apply<OutT><<<(unsigned)nb, kScanTPB, 0, s>>>(d_in, n, sums, d_out, d_total);
  cudaError_t e = cudaGetLastError();
  cudaFreeAsync(sums, s);
  if (e != cudaSuccess) return fail_cuda(e, "scan kernels");
  return GBO_OK;
}
}  // namespace

int exclusive_scan_i32(const int* d_in, int* d_out, long long n, long long* d_total,
                       cudaStream_t s) {
  return exclusive_scan<int>(d_in, d_out, n, d_total, s);
}

int exclusive_scan_i32_to_i64(const int* d_in, long long* d_out, long long n, long long* d_total,
                              cudaStream_t s) {
  return exclusive_scan<long long>(d_in, d_out, n, d_total, s);
}

// nnzb per block row: counts -> bsr_rowptr (device) and total (host).
static int nnzb_impl(const int* rowptr, const int* colind, int nrows, int ncols, long long nnz,
                     int b, int* bsr_rowptr, long long* h_total, cudaStream_t s) {
  const int nbr = (nrows + b - 1) / b;
  int* counts = nullptr;
  long long* d_total = nullptr;
  unsigned* derr = nullptr;
  GBO_CUDA_TRY(pool_malloc_async(&counts, sizeof(int) * (size_t)(nbr > 0 ? nbr : 1), s));
  GBO_CUDA_TRY(pool_malloc_async(&d_total, sizeof(long long) + sizeof(unsigned) * 2, s));
  derr = reinterpret_cast<unsigned*>(d_total + 1);
  GBO_CUDA_TRY(cudaMemsetAsync(derr, 0, sizeof(unsigned), s));
  int st = GBO_OK;
  if (nbr > 0) {
    st = dispatch_pack(b, false, rowptr, colind, nrows, ncols, nnz, nbr, counts, nullptr, nullptr,
                       nullptr, GBO_LAYOUT_ROW, derr, s);
    if (st == GBO_OK) st = exclusive_scan_i32(counts, bsr_rowptr, nbr, d_total, s);
  } else {
    GBO_CUDA_TRY(cudaMemsetAsync(bsr_rowptr, 0, sizeof(int), s));
    GBO_CUDA_TRY(cudaMemsetAsync(d_total, 0, sizeof(long long), s));
  }
  long long tot = 0;
  unsigned herr = 0;
  if (st == GBO_OK) {
    cudaError_t e1 = cudaMemcpyAsync(&tot, d_total, sizeof(long long), cudaMemcpyDeviceToHost, s);
    cudaError_t e2 = cudaMemcpyAsync(&herr, derr, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    cudaError_t e3 = cudaStreamSynchronize(s);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
      st = fail_cuda(e3 != cudaSuccess ? e3 : (e1 != cudaSuccess ? e1 : e2), "nnzb readback");
  }
  cudaFreeAsync(counts, s);
  cudaFreeAsync(d_total, s);
  if (st != GBO_OK) return st;
  GBO_TRY(derr_to_status(herr));
  if (tot > 2147483647LL) return fail(GBO_ERR_OVERFLOW, "more than 2^31-1 tiles; use a wider tile");
  *h_total = tot;
  return GBO_OK;
}

// Tile count of the B2SR packing of a device CSR at tile width b (the
// count pass of the packer alone; used by the tile-width tuner).
int count_tiles(const int* d_rowptr, const int* d_colind, int nrows, int ncols, long long nnz, int b,
                long long* nblk, cudaStream_t s) {
  const int nbr = (nrows + b - 1) / b;
  int* tmp = nullptr;
  GBO_CUDA_TRY(pool_malloc_async(&tmp, sizeof(int) * ((size_t)nbr + 1), s));
  const int st = nnzb_impl(d_rowptr, d_colind, nrows, ncols, nnz, b, tmp, nblk, s);
  cudaFreeAsync(tmp, s);
  return st;
}

static int fill_impl(const int* rowptr, const int* colind, int nrows, int ncols, long long nnz,
                     int b, int layout, const int* bsr_rowptr, int* bsr_colind, void* bsr_val,
                     cudaStream_t s, bool check) {
  const int nbr = (nrows + b - 1) / b;
  if (nbr == 0) return GBO_OK;
  unsigned* derr = nullptr;
  GBO_CUDA_TRY(pool_malloc_async(&derr, sizeof(unsigned), s));
  GBO_CUDA_TRY(cudaMemsetAsync(derr, 0, sizeof(unsigned), s));
  int st = dispatch_pack(b, true, rowptr, colind, nrows, ncols, nnz, nbr, nullptr, bsr_rowptr,
                         bsr_colind, bsr_val, layout, derr, s);
  unsigned herr = 0;
  if (st == GBO_OK && check) {
    cudaError_t e1 = cudaMemcpyAsync(&herr, derr, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    if (e1 != cudaSuccess || e2 != cudaSuccess) st = fail_cuda(e1 != cudaSuccess ? e1 : e2, "pack");
  }
  cudaFreeAsync(derr, s);
  if (st != GBO_OK) return st;
  return derr_to_status(herr);
}

int pack_into(gbo_graph* g, const int* d_rowptr, const int* d_colind, int nrows, int ncols,
              long long nnz, int b, int layout, cudaStream_t s) {
  g->nrows = nrows;
  g->ncols = ncols;
  g->b = b;
  g->layout = layout;
  g->nbr = (nrows + b - 1) / b;
  g->nbc = (ncols + b - 1) / b;
  g->nnz = nnz;
  GBO_CUDA_TRY(cudaMalloc(&g->rowptr, sizeof(int) * (size_t)(g->nbr + 1)));
  long long nblk = 0;
  GBO_TRY(nnzb_impl(d_rowptr, d_colind, nrows, ncols, nnz, b, g->rowptr, &nblk, s));
  g->nblk = nblk;
  size_t vb = (size_t)nblk * (size_t)b * (size_t)word_bytes(b);
  GBO_CUDA_TRY(cudaMalloc(&g->colind, sizeof(int) * (size_t)(nblk > 0 ? nblk : 1)));
  // pad the tile array to 16 bytes so vector loads past the end stay inside
  GBO_CUDA_TRY(cudaMalloc(&g->val, vb + 16));
  g->device_bytes += sizeof(int) * (g->nbr + 1) + sizeof(int) * nblk + vb + 16;
  GBO_TRY(fill_impl(d_rowptr, d_colind, nrows, ncols, nnz, b, layout, g->rowptr, g->colind,
                    g->val, s, false));
  return GBO_OK;
}

int compute_outdeg_from_cols(gbo_graph* g, const int* d_colind, long long nnz, int ncols,
                             cudaStream_t s) {
  GBO_CUDA_TRY(cudaMalloc(&g->outdeg, sizeof(int) * (size_t)(ncols > 0 ? ncols : 1)));
  GBO_CUDA_TRY(cudaMalloc(&g->invdeg, sizeof(float) * (size_t)(ncols > 0 ? ncols : 1)));
  g->device_bytes += 8LL * ncols;
  GBO_CUDA_TRY(cudaMemsetAsync(g->outdeg, 0, sizeof(int) * (size_t)ncols, s));
  if (nnz > 0) {
    unsigned grid = (unsigned)std::min<long long>((nnz + 255) / 256, 148LL * 64);
    k_col_hist<<<grid, 256, 0, s>>>(d_colind, nnz, ncols, g->outdeg);
  }
  if (ncols > 0) k_inv<<<blocks_for(ncols, 256), 256, 0, s>>>(g->outdeg, ncols, g->invdeg);
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

int compute_outdeg_from_rowptr(gbo_graph* g, const int* d_rowptr, int nrows, cudaStream_t s) {
  GBO_CUDA_TRY(cudaMalloc(&g->outdeg, sizeof(int) * (size_t)(nrows > 0 ? nrows : 1)));
  GBO_CUDA_TRY(cudaMalloc(&g->invdeg, sizeof(float) * (size_t)(nrows > 0 ? nrows : 1)));
  g->device_bytes += 8LL * nrows;
  if (nrows > 0) {
    k_row_len<<<blocks_for(nrows, 256), 256, 0, s>>>(d_rowptr, nrows, g->outdeg);
    k_inv<<<blocks_for(nrows, 256), 256, 0, s>>>(g->outdeg, nrows, g->invdeg);
  }
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

void launch_invdeg(const int* d_deg, int n, float* d_inv, cudaStream_t s) {
  if (n > 0) k_inv<<<blocks_for(n, 256), 256, 0, s>>>(d_deg, n, d_inv);
}

int upload_outdeg(gbo_graph* g, const int* h_deg, int n, cudaStream_t s) {
  GBO_CUDA_TRY(cudaMalloc(&g->outdeg, sizeof(int) * (size_t)(n > 0 ? n : 1)));
  GBO_CUDA_TRY(cudaMalloc(&g->invdeg, sizeof(float) * (size_t)(n > 0 ? n : 1)));
  g->device_bytes += 8LL * n;
  if (n > 0) {
    GBO_CUDA_TRY(cudaMemcpyAsync(g->outdeg, h_deg, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, s));
    launch_invdeg(g->outdeg, n, g->invdeg, s);
  }
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

int build_schedule(gbo_graph* g, cudaStream_t s) {
  const int nbr = g->nbr;
  g->chunk = chunk_for(g->b);
  if (nbr == 0) {
    g->nitems = 0;
    g->nsplit = 0;
    g->nslots = 0;
    return GBO_OK;
  }
  int *nchunk = nullptr, *nslot = nullptr, *issplit = nullptr;
  int *item_off = nullptr, *slot_off = nullptr, *split_off = nullptr;
  long long* tot = nullptr;
  size_t n1 = (size_t)nbr + 1;
  GBO_CUDA_TRY(pool_malloc_async(&nchunk, sizeof(int) * n1 * 6, s));
  nslot = nchunk + n1;
  issplit = nslot + n1;
  item_off = issplit + n1;
  slot_off = item_off + n1;
  split_off = slot_off + n1;
  GBO_CUDA_TRY(pool_malloc_async(&tot, sizeof(long long) * 3, s));
  k_sched_counts<<<blocks_for(nbr, 256), 256, 0, s>>>(g->rowptr, nbr, g->chunk, nchunk, nslot,
                                                      issplit);
  GBO_TRY(exclusive_scan_i32(nchunk, item_off, nbr, tot + 0, s));
  GBO_TRY(exclusive_scan_i32(nslot, slot_off, nbr, tot + 1, s));
  GBO_TRY(exclusive_scan_i32(issplit, split_off, nbr, tot + 2, s));
  long long h[3];
  GBO_CUDA_TRY(cudaMemcpyAsync(h, tot, sizeof(h), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  g->nitems = (int)h[0];
  g->nslots = (int)h[1];
  g->nsplit = (int)h[2];
  GBO_CUDA_TRY(cudaMalloc(&g->items, sizeof(gbo_item) * (size_t)(g->nitems > 0 ? g->nitems : 1)));
  GBO_CUDA_TRY(cudaMalloc(&g->splits, sizeof(gbo_split) * (size_t)(g->nsplit > 0 ? g->nsplit : 1)));
  g->device_bytes += sizeof(gbo_item) * (long long)g->nitems + sizeof(gbo_split) * (long long)g->nsplit;
  k_sched_fill<<<blocks_for(nbr, 256), 256, 0, s>>>(g->rowptr, nbr, g->chunk, item_off, slot_off,
                                                    split_off, g->items, g->splits);
  GBO_CUDA_TRY(cudaGetLastError());
  cudaFreeAsync(nchunk, s);
  cudaFreeAsync(tot, s);
  return GBO_OK;
}

// One warp per tile: bit r of the tile's occupancy word is set iff row word
// r is non-zero.  A 32x32 tile spans four 32-byte sectors while R-MAT-like
// graphs hold one or two set bits per tile, so pull kernels that read this
// word first and load only the non-empty row words move about half the
// bytes of a full tile read.
__global__ void k_rowmask32(const unsigned* __restrict__ val, long long nblk,
                            unsigned* __restrict__ mask) {
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nblk; t += nwarps) {
    const unsigned m = __ballot_sync(0xffffffffu, val[t * 32 + lane] != 0u);
    if (lane == 0) mask[t] = m;
  }
}

// Non-empty row words per work item (items cover the tiles in order).
__global__ void k_item_words(const gbo_item* __restrict__ items, int nitems,
                             const unsigned* __restrict__ mask, int* __restrict__ cnt) {
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nitems; i += nwarps) {
    const gbo_item it = items[i];
    int c = 0;
    for (int t = it.t0 + (int)lane; t < it.t1; t += 32) c += __popc(mask[t]);
    c = (int)__reduce_add_sync(0xffffffffu, (unsigned)c);
    if (lane == 0) cnt[i] = c;
  }
}

// Copy the non-empty row words of every tile, in tile order and row order
// inside a tile, to `out`; item i's words start at wbase[i].
__global__ void k_pack_rowwords(const gbo_item* __restrict__ items, int nitems,
                                const unsigned* __restrict__ val, const unsigned* __restrict__ mask,
                                const long long* __restrict__ wbase, unsigned* __restrict__ out) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nitems; i += nwarps) {
    const gbo_item it = items[i];
    long long base = wbase[i];
    for (int b0 = it.t0; b0 < it.t1; b0 += 32) {
      const int t = b0 + (int)lane;
      const unsigned m = t < it.t1 ? mask[t] : 0u;
      const int c = __popc(m);
      int incl = c;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if ((int)lane >= o) incl += y;
      }
      const int excl = incl - c;
      const int ntile = min(32, it.t1 - b0);
      for (int k0 = 0; k0 < ntile; k0 += 8) {  // eight tiles' words in flight
        unsigned w[8], mk[8];
        int ok[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          mk[u] = __shfl_sync(0xffffffffu, m, (k0 + u) & 31);
          ok[u] = __shfl_sync(0xffffffffu, excl, (k0 + u) & 31);
          if (k0 + u >= ntile) mk[u] = 0u;
          w[u] = (mk[u] >> lane) & 1u ? val[(size_t)(b0 + k0 + u) * 32 + lane] : 0u;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if ((mk[u] >> lane) & 1u) out[base + ok[u] + __popc(mk[u] & below)] = w[u];
      }
      base += __shfl_sync(0xffffffffu, incl, 31);
    }
  }
}

int build_rowwords(gbo_graph* g, cudaStream_t s) {
  if (!g->rowmask || g->rowword || g->nitems <= 0) return GBO_OK;
  int* cnt = nullptr;
  long long* tot = nullptr;
  GBO_CUDA_TRY(pool_malloc_async(&cnt, sizeof(int) * (size_t)g->nitems, s));
  GBO_CUDA_TRY(pool_malloc_async(&tot, sizeof(long long), s));
  GBO_CUDA_TRY(cudaMalloc(&g->item_wbase, sizeof(long long) * ((size_t)g->nitems + 1)));
  g->device_bytes += 8LL * (g->nitems + 1);
  int nsm = 148, dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (int)std::min<long long>(((long long)g->nitems + 7) / 8, 8LL * nsm);
  k_item_words<<<grid, 256, 0, s>>>(g->items, g->nitems, g->rowmask, cnt);
  GBO_TRY(exclusive_scan<long long>(cnt, g->item_wbase, g->nitems, tot, s));
  long long nw = 0;
  GBO_CUDA_TRY(cudaMemcpyAsync(&nw, tot, sizeof(nw), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  cudaFreeAsync(cnt, s);
  cudaFreeAsync(tot, s);
  GBO_CUDA_TRY(cudaMalloc(&g->rowword, sizeof(unsigned) * (size_t)(nw > 0 ? nw : 1)));
  g->nrowword = nw;
  g->device_bytes += 4LL * nw;
  k_pack_rowwords<<<grid, 256, 0, s>>>(g->items, g->nitems, static_cast<const unsigned*>(g->val),
                                       g->rowmask, g->item_wbase, g->rowword);
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

// Row-word slices, pass 1: warp per block row; per batch of 32 tiles (lane
// j: tile j's occupancy word) the number of tiles in which row r is
// non-empty is popc of the ballot of bit r, kept by lane r.  Writes the
// tail length max(count - kRwsHead, 0) of every padded row.
__global__ void k_rws_count(const int* __restrict__ rowptr, int nbr, const unsigned* __restrict__ mask,
                            int* __restrict__ tail_len) {
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long R = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; R < nbr; R += nwarps) {
    const int rs = rowptr[R], re = rowptr[R + 1];
    int c = 0;
    for (int t0 = rs; t0 < re; t0 += 32) {
      const unsigned m = t0 + (int)lane < re ? mask[t0 + lane] : 0u;
#pragma unroll
      for (int r = 0; r < 32; ++r) {
        const unsigned b = __ballot_sync(0xffffffffu, (m >> r) & 1u);
        if ((int)lane == r) c += __popc(b);
      }
    }
    tail_len[R * 32 + lane] = c > kRwsHead ? c - kRwsHead : 0;
  }
}

// Row-word slices, pass 2: warp per block row, lane r walks row r's word of
// every tile in order (one coalesced 128-byte load per tile, four tiles in
// flight) and appends the non-empty ones with their block column: the first
// kRwsHead to the head (entry-major), the rest to the row's tail.  Unused
// head entries get kRwsNone.
__global__ void k_rws_fill(const int* __restrict__ rowptr, const int* __restrict__ colind, int nbr,
                           const unsigned* __restrict__ val, const long long* __restrict__ tail_ptr,
                           uint2* __restrict__ head, uint2* __restrict__ tail) {
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long R = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; R < nbr; R += nwarps) {
    const int rs = rowptr[R], re = rowptr[R + 1];
    uint2* hp = head + (size_t)R * kRwsHead * 32 + lane;
    uint2* tp = tail + tail_ptr[R * 32 + lane];
    int k = 0;
    for (int t = rs; t < re; t += 4) {
      unsigned w[4];
      int c[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        w[u] = t + u < re ? val[(size_t)(t + u) * 32 + lane] : 0u;
        c[u] = t + u < re ? colind[t + u] : 0;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (!w[u]) continue;
        const uint2 e = make_uint2((unsigned)c[u], w[u]);
        if (k < kRwsHead) hp[(size_t)k * 32] = e;
        else tp[k - kRwsHead] = e;
        ++k;
      }
    }
    for (; k < kRwsHead; ++k) hp[(size_t)k * 32] = make_uint2(kRwsNone, 0u);
  }
}

int build_rws(gbo_graph* g, cudaStream_t s) {
  if (g->b != 32 || g->layout != GBO_LAYOUT_ROW || !g->rowmask || g->rws_head || g->nbr <= 0) return GBO_OK;
  const long long rows = (long long)g->nbr * 32;
  int* len = nullptr;
  long long* tot = nullptr;
  GBO_CUDA_TRY(pool_malloc_async(&len, sizeof(int) * (size_t)rows, s));
  GBO_CUDA_TRY(pool_malloc_async(&tot, sizeof(long long), s));
  GBO_CUDA_TRY(cudaMalloc(&g->rws_tail_ptr, sizeof(long long) * (size_t)(rows + 1)));
  GBO_CUDA_TRY(cudaMalloc(&g->rws_head, sizeof(uint2) * (size_t)rows * kRwsHead));
  g->device_bytes += 8LL * (rows + 1) + 8LL * rows * kRwsHead;
  int nsm = 148, dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (int)std::min<long long>(((long long)g->nbr + 7) / 8, 16LL * nsm);
  k_rws_count<<<grid, 256, 0, s>>>(g->rowptr, g->nbr, g->rowmask, len);
  GBO_TRY(exclusive_scan_i32_to_i64(len, g->rws_tail_ptr, rows, tot, s));
  long long nt = 0;
  GBO_CUDA_TRY(cudaMemcpyAsync(&nt, tot, sizeof(nt), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  cudaFreeAsync(len, s);
  cudaFreeAsync(tot, s);
  GBO_CUDA_TRY(cudaMalloc(&g->rws_tail, sizeof(uint2) * (size_t)(nt > 0 ? nt : 1)));
  g->rws_ntail = nt;
  g->device_bytes += 8LL * (nt > 0 ? nt : 1);
  k_rws_fill<<<grid, 256, 0, s>>>(g->rowptr, g->colind, g->nbr, static_cast<const unsigned*>(g->val),
                                  g->rws_tail_ptr, g->rws_head, g->rws_tail);
  GBO_CUDA_TRY(cudaGetLastError());
  // long tails cut into chunks (a host pass over the tail offsets, once)
  std::vector<long long> tp((size_t)rows + 1);
  GBO_CUDA_TRY(cudaMemcpyAsync(tp.data(), g->rws_tail_ptr, sizeof(long long) * tp.size(), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  std::vector<int> lrow, crow;
  std::vector<unsigned> lbits((size_t)g->nbr, 0u);
  std::vector<long long> lc0, cbeg, cend;
  for (long long i = 0; i < rows; ++i) {
    const long long len = tp[(size_t)i + 1] - tp[(size_t)i];
    if (len <= kRwsLongTail) continue;
    lrow.push_back((int)i);
    lbits[(size_t)(i / 32)] |= 1u << (31 - i % 32);
    lc0.push_back((long long)cbeg.size());
    for (long long b = tp[(size_t)i]; b < tp[(size_t)i + 1]; b += kRwsChunk) {
      crow.push_back((int)i);
      cbeg.push_back(b);
      cend.push_back(std::min(b + kRwsChunk, tp[(size_t)i + 1]));
    }
  }
  lc0.push_back((long long)cbeg.size());
  g->rws_nlong = (int)lrow.size();
  g->rws_nchunk = (long long)cbeg.size();
  auto up = [&](auto** dst, const auto& src) -> int {
    const size_t nb = sizeof(src[0]) * (src.empty() ? 1 : src.size());
    GBO_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(dst), nb));
    g->device_bytes += (long long)nb;
    if (!src.empty()) GBO_CUDA_TRY(cudaMemcpy(*dst, src.data(), nb, cudaMemcpyHostToDevice));
    return GBO_OK;
  };
  GBO_TRY(up(&g->rws_long_row, lrow));
  GBO_TRY(up(&g->rws_long_chunk0, lc0));
  GBO_TRY(up(&g->rws_chunk_row, crow));
  GBO_TRY(up(&g->rws_chunk_beg, cbeg));
  GBO_TRY(up(&g->rws_chunk_end, cend));
  GBO_TRY(up(&g->rws_longbits, lbits));
  return GBO_OK;
}

int build_rowmask(gbo_graph* g, cudaStream_t s) {
  if (g->b != 32 || g->layout != GBO_LAYOUT_ROW || g->rowmask) return GBO_OK;
  GBO_CUDA_TRY(cudaMalloc(&g->rowmask, sizeof(unsigned) * (size_t)(g->nblk > 0 ? g->nblk : 1)));
  g->device_bytes += 4LL * g->nblk;
  if (g->nblk > 0) {
    int nsm = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long long want = (g->nblk + 7) / 8;  // 8 warps per block
    const int grid = (int)std::min<long long>(want, 8LL * nsm);
    k_rowmask32<<<grid, 256, 0, s>>>(static_cast<const unsigned*>(g->val), g->nblk, g->rowmask);
  }
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

int ensure_workspace(gbo_graph* g, size_t bytes, cudaStream_t s) {
  if (g->ws_bytes >= bytes) return GBO_OK;
  if (g->ws) {
    GBO_CUDA_TRY(cudaStreamSynchronize(s));
    GBO_CUDA_TRY(cudaFree(g->ws));
    g->device_bytes -= (long long)g->ws_bytes;
    g->ws = nullptr;
    g->ws_bytes = 0;
  }
  size_t want = bytes + (bytes >> 3) + 256;
  GBO_CUDA_TRY(cudaMalloc(&g->ws, want));
  g->ws_bytes = want;
  g->device_bytes += (long long)want;
  return GBO_OK;
}

}  // namespace gbo

// ------------------------------------------------------------------ C ABI
using namespace gbo;

extern "C" int gbo_b2sr_nnzb(const int* d_csrRowPtr, const int* d_csrColInd, int nrows,
                             int ncols, int nnz, int tile_bits, int* d_bsrRowPtr, int* h_nblocks,
                             gbo_stream_t stream) {
  clear_error();
  if (!valid_tile_bits(tile_bits)) return fail(GBO_ERR_INVALID, "tile_bits must be 4, 8, 16, 32 or 64");
  if (nrows < 0 || ncols < 0 || nnz < 0 || !d_csrRowPtr || !d_bsrRowPtr || !h_nblocks ||
      (nnz > 0 && !d_csrColInd))
    return fail(GBO_ERR_INVALID, "gbo_b2sr_nnzb: bad argument");
  long long tot = 0;
  GBO_TRY(nnzb_impl(d_csrRowPtr, d_csrColInd, nrows, ncols, nnz, tile_bits, d_bsrRowPtr, &tot,
                    as_stream(stream)));
  *h_nblocks = (int)tot;
  return GBO_OK;
}

extern "C" int gbo_b2sr_pack(const int* d_csrRowPtr, const int* d_csrColInd, int nrows,
                             int ncols, int nnz, int tile_bits, int layout,
                             const int* d_bsrRowPtr, int* d_bsrColInd, void* d_bsrVal,
                             gbo_stream_t stream) {
  clear_error();
  if (!valid_tile_bits(tile_bits)) return fail(GBO_ERR_INVALID, "tile_bits must be 4, 8, 16, 32 or 64");
  if (layout != GBO_LAYOUT_ROW && layout != GBO_LAYOUT_COL)
    return fail(GBO_ERR_INVALID, "layout must be GBO_LAYOUT_ROW or GBO_LAYOUT_COL");
  if (nrows < 0 || ncols < 0 || nnz < 0 || !d_csrRowPtr || !d_bsrRowPtr ||
      (nnz > 0 && (!d_csrColInd || !d_bsrColInd || !d_bsrVal)))
    return fail(GBO_ERR_INVALID, "gbo_b2sr_pack: bad argument");
  return fill_impl(d_csrRowPtr, d_csrColInd, nrows, ncols, nnz, tile_bits, layout, d_bsrRowPtr,
                   d_bsrColInd, d_bsrVal, as_stream(stream), true);
}

template <int B>
static int pack_vec_impl(const float* xf, const int32_t* xi, int n, void* bits, cudaStream_t s) {
  long long nw = ((long long)n + B - 1) / B;
  if (B == 64) GBO_CUDA_TRY(cudaMemsetAsync(bits, 0, sizeof(unsigned long long) * nw, s));
  long long threads = ((long long)n + 31) / 32 * 32;
  if (B == 64) threads = nw * 64;  // whole 64-element words
  if (threads == 0) return GBO_OK;
  k_pack_vec<B><<<blocks_for(threads, 256), 256, 0, s>>>(
      xf, xi, n, reinterpret_cast<typename Word<B>::T*>(bits), nw);
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

static int pack_vec_dispatch(const float* xf, const int32_t* xi, int n, int b, void* bits,
                             gbo_stream_t stream) {
  clear_error();
  if (!valid_tile_bits(b)) return fail(GBO_ERR_INVALID, "tile_bits must be 4, 8, 16, 32 or 64");
  if (n < 0 || (n > 0 && (!bits || (!xf && !xi)))) return fail(GBO_ERR_INVALID, "pack_vector: bad argument");
  cudaStream_t s = as_stream(stream);
  switch (b) {
    case 4: return pack_vec_impl<4>(xf, xi, n, bits, s);
    case 8: return pack_vec_impl<8>(xf, xi, n, bits, s);
    case 16: return pack_vec_impl<16>(xf, xi, n, bits, s);
    case 32: return pack_vec_impl<32>(xf, xi, n, bits, s);
    default: return pack_vec_impl<64>(xf, xi, n, bits, s);
  }
}

extern "C" int gbo_pack_vector_f32(const float* d_x, int n, int tile_bits, void* d_bits,
                                   gbo_stream_t stream) {
  return pack_vec_dispatch(d_x, nullptr, n, tile_bits, d_bits, stream);
}
extern "C" int gbo_pack_vector_i32(const int32_t* d_x, int n, int tile_bits, void* d_bits,
                                   gbo_stream_t stream) {
  return pack_vec_dispatch(nullptr, d_x, n, tile_bits, d_bits, stream);
}

extern "C" int gbo_unpack_vector(const void* d_bits, int n, int tile_bits, int32_t* d_out,
                                 gbo_stream_t stream) {
  clear_error();
  if (!valid_tile_bits(tile_bits)) return fail(GBO_ERR_INVALID, "tile_bits must be 4, 8, 16, 32 or 64");
  if (n < 0 || (n > 0 && (!d_bits || !d_out))) return fail(GBO_ERR_INVALID, "unpack_vector: bad argument");
  if (n == 0) return GBO_OK;
  cudaStream_t s = as_stream(stream);
  unsigned grid = blocks_for(n, 256);
  switch (tile_bits) {
    case 4: k_unpack_vec<4><<<grid, 256, 0, s>>>((const uint8_t*)d_bits, n, d_out); break;
    case 8: k_unpack_vec<8><<<grid, 256, 0, s>>>((const uint8_t*)d_bits, n, d_out); break;
    case 16: k_unpack_vec<16><<<grid, 256, 0, s>>>((const uint16_t*)d_bits, n, d_out); break;
    case 32: k_unpack_vec<32><<<grid, 256, 0, s>>>((const uint32_t*)d_bits, n, d_out); break;
    default: k_unpack_vec<64><<<grid, 256, 0, s>>>((const unsigned long long*)d_bits, n, d_out); break;
  }
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

extern "C" int gbo_invdeg_from_rowptr(const int* d_rowptr, int n, float* d_inv, gbo_stream_t stream) {
  clear_error();
  if (n < 0 || (n > 0 && (!d_rowptr || !d_inv))) return fail(GBO_ERR_INVALID, "invdeg: bad argument");
  if (n == 0) return GBO_OK;
  cudaStream_t s = as_stream(stream);
  int* deg = nullptr;
  GBO_CUDA_TRY(pool_malloc_async(&deg, sizeof(int) * (size_t)n, s));
  k_row_len<<<blocks_for(n, 256), 256, 0, s>>>(d_rowptr, n, deg);
  k_inv<<<blocks_for(n, 256), 256, 0, s>>>(deg, n, d_inv);
  cudaError_t e = cudaGetLastError();
  cudaFreeAsync(deg, s);
  if (e != cudaSuccess) return fail_cuda(e, "invdeg kernels");
  return GBO_OK;
}
