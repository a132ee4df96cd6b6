// Matrix Market ingestion on the GPU: the entry lines are parsed in parallel
// and the CSR is built in device memory, with the semantics of the host
// reader gbo_read_mtx -- readMtx + coo2csr (algorithm/readMtx.hpp:351-423,
// 246-304) or mmio_data (algorithm/mmio_highlevel.h:139-309).  The
// reference parses with fscanf one entry at a time and sorts a vector of
// tuples on the host, the wall-time bottleneck before its kernels.
//
// The banner, comments and size line are parsed on the host; the bytes after
// them go to the device, where
//   1. every line start is found (a thread per 16 bytes, positions sorted),
//   2. a thread per line skips blanks and parses "i j" (lines without a
//      number are blank; the first nnz non-blank lines are the entries),
//   3. the (row, col) pairs -- mirrored as the mode says, self-loops dropped
//      for readMtx -- are sorted as 64-bit keys (CUB radix sort), duplicates
//      dropped for readMtx, and the row offsets come from a histogram + scan.
// Result: the same CSR as the host reader (rows ascending, columns ascending
// inside a row).
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include <cub/cub.cuh>

#include "graph.cuh"
#include "host_common.h"

namespace gbo {
namespace {

enum : unsigned { MTX_MALFORMED = 1u, MTX_BOUNDS = 2u };

__device__ __forceinline__ bool blank(unsigned char ch) {
  return ch == ' ' || ch == '\t' || ch == '\r' || ch == '\v' || ch == '\f';
}

// Newlines of the section (16 bytes per thread), to size the line list.
__global__ void k_count_newlines(const unsigned char* __restrict__ s, long long n,
                                 unsigned long long* __restrict__ count) {
  unsigned c = 0;
  const long long step = (long long)gridDim.x * blockDim.x * 16;
  for (long long i0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 16; i0 < n; i0 += step) {
    const long long i1 = i0 + 16 < n ? i0 + 16 : n;
    for (long long i = i0; i < i1; ++i) c += s[i] == '\n';
  }
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// Line starts: position 0 and every position after a '\n' (16 bytes per
// thread), appended through a counter; sorted afterwards.
__global__ void k_line_starts(const unsigned char* __restrict__ s, long long n,
                              long long* __restrict__ starts, unsigned long long* __restrict__ count) {
  const long long step = (long long)gridDim.x * blockDim.x * 16;
  for (long long i0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 16; i0 < n; i0 += step) {
    if (i0 == 0) starts[atomicAdd(count, 1ull)] = 0;
    const long long i1 = i0 + 16 < n ? i0 + 16 : n;
    for (long long i = i0; i < i1; ++i)
      if (s[i] == '\n' && i + 1 < n) starts[atomicAdd(count, 1ull)] = i + 1;
  }
}

// Parse a decimal integer with an optional sign at s[*p]; false if no digit.
__device__ __forceinline__ bool parse_int(const unsigned char* __restrict__ s, long long n, long long* p,
                                          long long* out) {
  long long q = *p;
  bool neg = false;
  if (q < n && (s[q] == '+' || s[q] == '-')) {
    neg = s[q] == '-';
    ++q;
  }
  long long v = 0;
  int digits = 0;
  while (q < n && s[q] >= '0' && s[q] <= '9') {
    if (digits < 19) v = v * 10 + (s[q] - '0');
    ++digits;
    ++q;
  }
  if (digits == 0) return false;
  if (digits > 18) v = (long long)9e18;  // far outside any matrix
  *out = neg ? -v : v;
  *p = q;
  return true;
}

// A thread per line: is it blank, and if not its "i j" (1-based, checked).
__global__ void k_parse_lines(const unsigned char* __restrict__ s, long long n,
                              const long long* __restrict__ starts, long long nlines, long long nrows,
                              long long ncols, int* __restrict__ nonblank, int* __restrict__ I,
                              int* __restrict__ J, unsigned* __restrict__ err) {
  for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < nlines;
       l += (long long)gridDim.x * blockDim.x) {
    long long p = starts[l];
    while (p < n && blank(s[p])) ++p;
    if (p >= n || s[p] == '\n') {
      nonblank[l] = 0;
      continue;
    }
    nonblank[l] = 1;
    long long i = 0, j = 0;
    if (!parse_int(s, n, &p, &i)) {
      I[l] = -1;  // reported only if this line is one of the entries
      J[l] = -1;
      continue;
    }
    while (p < n && blank(s[p])) ++p;
    if (!parse_int(s, n, &p, &j)) j = 0;
    const bool ok = i >= 1 && j >= 1 && i <= nrows && j <= ncols;
    I[l] = ok ? (int)(i - 1) : -2;
    J[l] = ok ? (int)(j - 1) : -2;
  }
}

// Entries: the first nnz non-blank lines (ranks from an exclusive scan).
// Writes the pairs -- and, where asked, the mirrored off-diagonal pairs
// after the first nnz -- as keys row << 32 | col; a dropped pair gets the
// key ~0 (sorted to the end and cut off).
__global__ void k_entry_keys(const int* __restrict__ nonblank, const long long* __restrict__ rank,
                             const int* __restrict__ I, const int* __restrict__ J, long long nlines,
                             long long nnz, bool mirror, bool drop_self,
                             unsigned long long* __restrict__ keys, unsigned* __restrict__ err) {
  for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < nlines;
       l += (long long)gridDim.x * blockDim.x) {
    if (!nonblank[l]) continue;
    const long long k = rank[l];
    if (k >= nnz) continue;
    const int i = I[l], j = J[l];
    if (i == -1) {
      atomicOr(err, MTX_MALFORMED);
      continue;
    }
    if (i < 0) {
      atomicOr(err, MTX_BOUNDS);
      continue;
    }
    const unsigned long long none = ~0ull;
    const bool self = i == j;
    keys[k] = drop_self && self ? none : ((unsigned long long)i << 32) | (unsigned)j;
    if (mirror) keys[nnz + k] = self ? none : ((unsigned long long)j << 32) | (unsigned)i;
  }
}

__global__ void k_row_hist(const unsigned long long* __restrict__ keys, long long m, int* __restrict__ cnt,
                           int* __restrict__ colind) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < m;
       k += (long long)gridDim.x * blockDim.x) {
    const unsigned long long key = keys[k];
    atomicAdd(cnt + (key >> 32), 1);
    colind[k] = (int)(key & 0xffffffffull);
  }
}

// Stream-ordered scratch, freed on scope exit.
struct DevMem {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  explicit DevMem(cudaStream_t st) : s(st) {}
  ~DevMem() {
    if (p) cudaFreeAsync(p, s);
  }
  int alloc(size_t bytes) {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    GBO_CUDA_TRY(pool_malloc_async(&p, bytes ? bytes : 1, s));
    return GBO_OK;
  }
};

unsigned grid_for(long long n, int per_thread = 1) {
  const long long t = (n + per_thread - 1) / per_thread;
  return (unsigned)std::max<long long>(1, std::min<long long>((t + 255) / 256, 1ll << 20));
}

}  // namespace

// Parse `path` on the GPU into a device CSR (rowptr int32[nrows+1], colind
// int32[nnz]) allocated with cudaMalloc.
static int read_mtx_device(const char* path, int mode, int directed, int** d_rowptr, int** d_colind, int* nrows,
                    int* ncols, long long* nnz_out, cudaStream_t s) {
  FILE* f = fopen(path, "rb");
  if (!f) return fail(GBO_ERR_IO, std::string("cannot read ") + path);
  fseek(f, 0, SEEK_END);
  const long long size = ftell(f);
  fseek(f, 0, SEEK_SET);
  // pageable host copy of the file (pinning it would cost more than the
  // staged transfer saves)
  std::vector<char> text((size_t)std::max(size, 0ll) + 1);
  char* h = text.data();
  const size_t got = size > 0 ? fread(h, 1, (size_t)size, f) : 0;
  fclose(f);
  if ((long long)got != size) return fail(GBO_ERR_IO, std::string("cannot read ") + path);
  h[size] = '\0';
  MtxHeader hd;
  const char* entries = nullptr;
  GBO_TRY(parse_mtx_header(h, h + size, &hd, &entries));
  const long long off = entries - h, n = size - off, z = hd.nnz;
  bool mirror, drop_self, dedup;
  if (mode == GBO_MTX_READMTX) {
    // undirected if the banner says symmetric or directed == 2, never if
    // directed == 1 (readMtx.hpp:380-384)
    mirror = (hd.symmetric || directed == 2) && directed != 1;
    drop_self = env_remove_self_loops();
    dedup = true;
  } else {
    mirror = hd.symmetric || hd.hermitian;  // mmio_highlevel.h:213-292
    drop_self = false;
    dedup = false;
  }
  // the entry section on the device
  DevMem dtext(s), dstarts(s), dcount(s);
  GBO_TRY(dtext.alloc((size_t)std::max(n, 1ll)));
  if (n > 0) GBO_CUDA_TRY(cudaMemcpyAsync(dtext.p, h + off, (size_t)n, cudaMemcpyHostToDevice, s));
  const auto* ds = static_cast<const unsigned char*>(dtext.p);
  // 1. line starts (one after every newline, plus the first)
  GBO_TRY(dcount.alloc(sizeof(unsigned long long) + sizeof(unsigned)));
  auto* dcnt = static_cast<unsigned long long*>(dcount.p);
  auto* dE = reinterpret_cast<unsigned*>(dcnt + 1);
  GBO_CUDA_TRY(cudaMemsetAsync(dcount.p, 0, sizeof(unsigned long long) + sizeof(unsigned), s));
  unsigned long long newlines = 0;
  if (n > 0) k_count_newlines<<<grid_for(n, 16), 256, 0, s>>>(ds, n, dcnt);
  GBO_CUDA_TRY(cudaMemcpyAsync(&newlines, dcnt, sizeof(newlines), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaMemsetAsync(dcnt, 0, sizeof(unsigned long long), s));
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  GBO_TRY(dstarts.alloc(sizeof(long long) * ((size_t)newlines + 1)));
  auto* starts = static_cast<long long*>(dstarts.p);
  if (n > 0) k_line_starts<<<grid_for(n, 16), 256, 0, s>>>(ds, n, starts, dcnt);
  unsigned long long nl = 0;
  GBO_CUDA_TRY(cudaMemcpyAsync(&nl, dcnt, sizeof(nl), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  const long long nlines = (long long)nl;
  if (nlines > 2147483647LL) return fail(GBO_ERR_OVERFLOW, "more than 2^31-1 lines");
  // sort the line starts
  DevMem sorted(s), temp(s);
  GBO_TRY(sorted.alloc(sizeof(long long) * (size_t)std::max(nlines, 1ll)));
  size_t tb = 0;
  GBO_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tb, (const unsigned long long*)nullptr,
                                              (unsigned long long*)nullptr, (int)nlines, 0, 64, s));
  GBO_TRY(temp.alloc(tb));
  if (nlines > 0)
    GBO_CUDA_TRY(cub::DeviceRadixSort::SortKeys(temp.p, tb, reinterpret_cast<const unsigned long long*>(starts),
                                                static_cast<unsigned long long*>(sorted.p), (int)nlines, 0, 64, s));
  // 2. parse every line
  DevMem nb(s), rank(s), dI(s), dJ(s), tot(s);
  GBO_TRY(nb.alloc(sizeof(int) * (size_t)std::max(nlines, 1ll)));
  GBO_TRY(rank.alloc(sizeof(long long) * ((size_t)nlines + 1)));
  GBO_TRY(dI.alloc(sizeof(int) * (size_t)std::max(nlines, 1ll)));
  GBO_TRY(dJ.alloc(sizeof(int) * (size_t)std::max(nlines, 1ll)));
  GBO_TRY(tot.alloc(sizeof(long long)));
  if (nlines > 0)
    k_parse_lines<<<grid_for(nlines), 256, 0, s>>>(ds, n, static_cast<const long long*>(sorted.p), nlines,
                                                   hd.nrows, hd.ncols, static_cast<int*>(nb.p),
                                                   static_cast<int*>(dI.p), static_cast<int*>(dJ.p), dE);
  GBO_TRY(exclusive_scan_i32_to_i64(static_cast<int*>(nb.p), static_cast<long long*>(rank.p), nlines,
                                    static_cast<long long*>(tot.p), s));
  long long nonblank = 0;
  GBO_CUDA_TRY(cudaMemcpyAsync(&nonblank, tot.p, sizeof(nonblank), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  if (nonblank < z) return fail(GBO_ERR_IO, "fewer entries than the size line promises");
  // 3. keys, sort, dedup, CSR
  const long long m = mirror ? 2 * z : z;
  DevMem keys(s), keys2(s);
  GBO_TRY(keys.alloc(sizeof(unsigned long long) * (size_t)std::max(m, 1ll)));
  GBO_TRY(keys2.alloc(sizeof(unsigned long long) * (size_t)std::max(m, 1ll)));
  auto* k0 = static_cast<unsigned long long*>(keys.p);
  auto* k1 = static_cast<unsigned long long*>(keys2.p);
  if (nlines > 0)
    k_entry_keys<<<grid_for(nlines), 256, 0, s>>>(static_cast<const int*>(nb.p),
                                                  static_cast<const long long*>(rank.p),
                                                  static_cast<const int*>(dI.p), static_cast<const int*>(dJ.p),
                                                  nlines, z, mirror, drop_self, k0, dE);
  unsigned herr = 0;
  GBO_CUDA_TRY(cudaMemcpyAsync(&herr, dE, sizeof(herr), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  if (herr & MTX_MALFORMED) return fail(GBO_ERR_IO, "malformed entry line");
  if (herr & MTX_BOUNDS) return fail(GBO_ERR_BOUNDS, "entry index outside the matrix");
  if (m > 2147483647LL) return fail(GBO_ERR_OVERFLOW, "more than 2^31-1 entries");
  tb = 0;
  GBO_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tb, k0, k1, (int)m, 0, 64, s));
  size_t tb2 = 0;
  GBO_CUDA_TRY(cub::DeviceSelect::Unique(nullptr, tb2, k1, k0, dcnt, (int)m, s));
  GBO_TRY(temp.alloc(std::max(tb, tb2)));
  long long kept = m;
  const unsigned long long* sk = k1;
  if (m > 0) {
    GBO_CUDA_TRY(cub::DeviceRadixSort::SortKeys(temp.p, tb, k0, k1, (int)m, 0, 64, s));
    if (dedup) {
      tb2 = std::max(tb, tb2);
      GBO_CUDA_TRY(cub::DeviceSelect::Unique(temp.p, tb2, k1, k0, dcnt, (int)m, s));
      sk = k0;
      unsigned long long u = 0;
      GBO_CUDA_TRY(cudaMemcpyAsync(&u, dcnt, sizeof(u), cudaMemcpyDeviceToHost, s));
      GBO_CUDA_TRY(cudaStreamSynchronize(s));
      kept = (long long)u;
    }
    // dropped pairs (key ~0) sort last: cut them off
    std::vector<unsigned long long> tail(1);
    long long lo = 0, hi = kept;  // first index whose key is ~0
    while (lo < hi) {
      const long long mid = (lo + hi) / 2;
      GBO_CUDA_TRY(cudaMemcpy(tail.data(), sk + mid, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
      if (tail[0] == ~0ull) hi = mid;
      else lo = mid + 1;
    }
    kept = lo;
  }
  int *rp = nullptr, *ci = nullptr;
  GBO_CUDA_TRY(cudaMalloc(&rp, sizeof(int) * ((size_t)hd.nrows + 1)));
  if (cudaMalloc(&ci, sizeof(int) * (size_t)std::max(kept, 1ll)) != cudaSuccess) {
    cudaFree(rp);
    return fail(GBO_ERR_NOMEM, "CSR columns");
  }
  DevMem rowcnt(s);
  int st = rowcnt.alloc(sizeof(int) * (size_t)std::max(hd.nrows, 1));
  if (st == GBO_OK && hd.nrows > 0 && cudaMemsetAsync(rowcnt.p, 0, sizeof(int) * (size_t)hd.nrows, s) != cudaSuccess)
    st = fail(GBO_ERR_CUDA, "memset");
  if (st == GBO_OK && kept > 0) k_row_hist<<<grid_for(kept), 256, 0, s>>>(sk, kept, static_cast<int*>(rowcnt.p), ci);
  if (st == GBO_OK) st = exclusive_scan_i32(static_cast<int*>(rowcnt.p), rp, hd.nrows, static_cast<long long*>(tot.p), s);
  if (st == GBO_OK && cudaStreamSynchronize(s) != cudaSuccess) st = fail(GBO_ERR_CUDA, "CSR build");
  if (st != GBO_OK) {
    cudaFree(rp);
    cudaFree(ci);
    return st;
  }
  *d_rowptr = rp;
  *d_colind = ci;
  *nrows = hd.nrows;
  *ncols = hd.ncols;
  *nnz_out = kept;
  return GBO_OK;
}

}  // namespace gbo

using namespace gbo;

extern "C" int gbo_read_mtx_device(const char* path, int mode, int directed, int** d_rowptr, int** d_colind,
                                   int* nrows, int* ncols, int64_t* nnz, gbo_stream_t stream) {
  clear_error();
  if (!path || !d_rowptr || !d_colind || !nrows || !ncols || !nnz) return fail(GBO_ERR_INVALID, "NULL argument");
  if (mode != GBO_MTX_READMTX && mode != GBO_MTX_MMIO) return fail(GBO_ERR_INVALID, "bad mode");
  long long z = 0;
  GBO_TRY(read_mtx_device(path, mode, directed, d_rowptr, d_colind, nrows, ncols, &z, as_stream(stream)));
  *nnz = z;
  return GBO_OK;
}

extern "C" int gbo_graph_from_mtx(const char* path, int mode, int directed, int tile_bits, int flags,
                                  gbo_stream_t stream, gbo_graph** out) {
  clear_error();
  if (!path || !out) return fail(GBO_ERR_INVALID, "NULL argument");
  if (mode != GBO_MTX_READMTX && mode != GBO_MTX_MMIO) return fail(GBO_ERR_INVALID, "bad mode");
  int *rp = nullptr, *ci = nullptr, nr = 0, nc = 0;
  long long z = 0;
  cudaStream_t s = as_stream(stream);
  GBO_TRY(read_mtx_device(path, mode, directed, &rp, &ci, &nr, &nc, &z, s));
  const int st = gbo_graph_from_csr(rp, ci, nr, nc, (int)z, tile_bits, flags | GBO_FLAG_DEVICE_PTRS, stream, out);
  cudaStreamSynchronize(s);
  cudaFree(rp);
  cudaFree(ci);
  return st;
}
